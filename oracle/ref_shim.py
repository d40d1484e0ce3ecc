"""Generate the globals translation unit for the reference's host files.

The reference defines most process globals in src/bluebottle.c, which
cannot be compiled here (it needs MPI); src/particle.c defines its own.
This script turns every single-line `extern` variable declaration of
src/bluebottle.h and src/recorder.h into a definition, so that
src/domain.c, src/particle.c and src/rng.c link into a shared library of
their own under oracle/_ref/.  Run by oracle/ref.mk:

  python oracle/ref_shim.py REFERENCE_SRC_DIR OUT.c
"""
import os
import re
import sys

HEADERS = ("bluebottle.h", "recorder.h")


def main():
    src, out = sys.argv[1], sys.argv[2]
    seen = set()
    lines = ['#include "bluebottle.h"', '#include "particle.h"',
             '#include "recorder.h"', ""]
    for h in HEADERS:
        path = os.path.join(src, h)
        if not os.path.exists(path):
            continue
        for ln in open(path):
            m = re.match(r"^\s*extern\s+([^(;\"]+);\s*$", ln)
            if not m:
                continue
            decl = m.group(1).strip()
            name = re.findall(r"(\w+)\s*(?:\[[^\]]*\])*\s*$", decl)
            if not name or name[0] in seen:
                continue
            seen.add(name[0])
            lines.append(decl + ";")
    with open(out, "w") as fh:
        fh.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
