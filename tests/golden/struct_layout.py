"""Struct layouts (sizeof, and offsetof of every field) of the structs the
C ABI shares with the reference: grid_info, dom_struct (src/domain.h),
g_struct, gradP_struct, BC (src/bluebottle.h), cage_struct, part_struct
(src/particle.h).

  python tests/golden/struct_layout.py REFERENCE_SRC_DIR

compiles a probe against the reference's own headers (with an empty
cgnslib.h stub, -DDOUBLE) and writes ref_struct_layout.json beside this
file.  The tests call layout_of() on this repository's header and compare.
The field lists are those of bluebottle_b200.abi's ctypes mirrors.
"""
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from bluebottle_b200 import abi  # noqa: E402

STRUCTS = [("grid_info", abi.GridInfo), ("dom_struct", abi.DomStruct),
           ("g_struct", abi.GStruct), ("gradP_struct", abi.GStruct),
           ("BC", abi.BCStruct), ("cage_struct", abi.CageStruct),
           ("part_struct", abi.PartStruct)]


def probe_source(include_line):
    lines = [include_line, "#include <stdio.h>", "#include <stddef.h>",
             "int main(void) {", '  printf("{");']
    first = True
    for cname, cls in STRUCTS:
        sep = "" if first else ","
        first = False
        lines.append('  printf("%s\\"%s\\": {\\"sizeof\\": %%zu", sizeof(%s));'
                     % (sep, cname, cname))
        for fname, _ in cls._fields_:
            lines.append('  printf(", \\"%s\\": %%zu", offsetof(%s, %s));'
                         % (fname, cname, fname))
        lines.append('  printf("}");')
    lines += ['  printf("}\\n");', "  return 0;", "}"]
    return "\n".join(lines) + "\n"


def layout_of(include_dirs, include_line, defines=("DOUBLE",)):
    with tempfile.TemporaryDirectory() as tmp:
        open(os.path.join(tmp, "cgnslib.h"), "w").close()
        src = os.path.join(tmp, "probe.c")
        exe = os.path.join(tmp, "probe")
        with open(src, "w") as fh:
            fh.write(probe_source(include_line))
        cmd = ["gcc", "-std=gnu99", "-fopenmp", "-o", exe, src, "-I" + tmp]
        cmd += ["-I" + d for d in include_dirs]
        cmd += ["-D" + d for d in defines]
        subprocess.run(cmd, check=True, capture_output=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True)
        return json.loads(out.stdout)


def main():
    ref_src = sys.argv[1]
    lay = layout_of([ref_src], '#include "particle.h"')
    with open(os.path.join(HERE, "ref_struct_layout.json"), "w") as fh:
        json.dump(lay, fh, indent=1, sort_keys=True)
        fh.write("\n")
    print("wrote", os.path.join(HERE, "ref_struct_layout.json"))


if __name__ == "__main__":
    main()
