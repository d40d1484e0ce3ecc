"""The C-ABI boundary without a GPU: the library loads, exports every
function include/*.h declares, and shares struct layouts with the
reference's headers (golden layouts in tests/golden/ref_struct_layout.json,
made by tests/golden/struct_layout.py from src/domain.h, src/bluebottle.h,
src/particle.h)."""
import ctypes as C
import json
import os
import re

import pytest

from bluebottle_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def declared_functions():
    """Function names declared at file scope in include/*.h."""
    names = set()
    for fn in sorted(os.listdir(INCLUDE)):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, fn)).read()
        text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
        text = re.sub(r"//[^\n]*", " ", text)
        text = re.sub(r"^\s*#.*$", " ", text, flags=re.M)
        # drop struct bodies and typedefs
        text = re.sub(r"typedef\s+struct[^{;]*\{.*?\}\s*\w+\s*;", " ", text, flags=re.S)
        text = re.sub(r"extern\s+\"C\"\s*\{|\}", " ", text)
        for stmt in text.split(";"):
            stmt = " ".join(stmt.split())
            if not stmt or stmt.startswith("extern ") and "(" not in stmt:
                continue
            m = re.match(r"^(?:extern\s+)?[\w\s\*]+?\b(\w+)\s*\(", stmt)
            if m and not stmt.startswith("typedef"):
                names.add(m.group(1))
    return names


def test_header_parse_finds_entry_points():
    names = declared_functions()
    for must in ("cuda_PP_bicgstab", "cuda_build_cages", "cuda_Lamb",
                 "cuda_move_parts", "bbb_step", "bbb_PP_bicgstab_static"):
        assert must in names


def test_library_exports_every_declared_function():
    lib = abi.load()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert missing == []


def test_ctypes_mirror_declares_every_header_function():
    assert sorted(declared_functions() - set(abi.DECLARED)) == []


def test_reference_globals_exported():
    """The reference's host globals the entry points read (src/bluebottle.c
    :29-187) exist in the library, weak, so bluebottle.c's win at link."""
    lib = abi.load()
    for g in ("dom", "Dom", "bc", "parts", "dt", "dt0", "ttime", "nu", "mu",
              "rho_f", "g", "gradP", "pp_max_iter", "pp_residual",
              "lamb_relax", "lamb_cut", "out_plane", "nparts", "coeff_stride",
              "p", "p0", "phi", "u", "v", "w", "u0", "v0", "w0"):
        C.c_int.in_dll(lib, g)      # raises ValueError when absent


def _golden_layout():
    with open(os.path.join(GOLDEN, "ref_struct_layout.json")) as fh:
        return json.load(fh)


def test_header_struct_layout_matches_reference():
    import sys
    sys.path.insert(0, GOLDEN)
    from struct_layout import layout_of
    ours = layout_of([INCLUDE], '#include "bluebottle_b200_types.h"')
    assert ours == _golden_layout()


@pytest.mark.parametrize("cname,cls", [
    ("grid_info", abi.GridInfo), ("dom_struct", abi.DomStruct),
    ("g_struct", abi.GStruct), ("BC", abi.BCStruct),
    ("cage_struct", abi.CageStruct), ("part_struct", abi.PartStruct)])
def test_ctypes_layout_matches_reference(cname, cls):
    ref = _golden_layout()[cname]
    assert C.sizeof(cls) == ref["sizeof"]
    for fname, _ in cls._fields_:
        assert getattr(cls, fname).offset == ref[fname], fname


def test_status_strings():
    lib = abi.load()
    for code in range(0, 9):
        s = lib.bbb_status_string(code)
        assert s and len(s) >= 2
    assert lib.bbb_device_count() >= 0


@pytest.mark.parametrize("cname,cls", [("bbb_stats", abi.Stats),
                                       ("bbb_options", abi.Options)])
def test_library_struct_mirrors_match_header(cname, cls, tmp_path):
    """The ctypes mirrors of the library's own structs (statistics, options)
    against the header, compiled: every field's offset and the size."""
    import json
    import subprocess
    lines = ['#include "bluebottle_b200.h"', "#include <stdio.h>",
             "#include <stddef.h>", "int main(void) {",
             '  printf("{\\"sizeof\\": %%zu", sizeof(%s));' % cname]
    for fname, _ in cls._fields_:
        lines.append('  printf(", \\"%s\\": %%zu", offsetof(%s, %s));'
                     % (fname, cname, fname))
    lines += ['  printf("}\\n");', "  return 0;", "}"]
    src, exe = tmp_path / "probe.c", tmp_path / "probe"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=gnu99", "-o", str(exe), str(src), "-I" + INCLUDE],
                   check=True, capture_output=True)
    got = json.loads(subprocess.run([str(exe)], check=True, capture_output=True,
                                    text=True).stdout)
    assert C.sizeof(cls) == got["sizeof"]
    for fname, _ in cls._fields_:
        assert getattr(cls, fname).offset == got[fname], fname
