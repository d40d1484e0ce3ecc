"""Child process of test_dropin.py: the reference's own host files
(src/domain.c, src/particle.c, src/rng.c, src/vtk.c, linked against
libbbb200.so into oracle/_ref/libref_dropin.so) set up and write out the
state of this library, as src/bluebottle.c's program does.

usage: python dropin_child.py RUNDIR MODE OUT.npz
  MODE ref   -- set up with the reference's readers and initialisers
  MODE ours  -- set up with the library's own (bbb_read_input, ...)
  MODE refrun / oursrun -- the same, then two GPU steps and a pull
Every mode then fills p with a known pattern where it has not run, calls
the reference's out_VTK, and saves the host state and the VTK pressure."""
import ctypes as C
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from bluebottle_b200 import abi  # noqa: E402

FACE = {"u": "Gfx", "v": "Gfy", "w": "Gfz", "u0": "Gfx", "conv0_w": "Gfz"}
CELL = ("p", "p0", "phi")


def main():
    run, mode, out = sys.argv[1], sys.argv[2], sys.argv[3]
    lib = abi.load()
    ref = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_dropin.so"),
                 mode=C.RTLD_GLOBAL)
    os.chdir(run)
    lib.bbb_set_exit_on_failure(0)
    if mode.startswith("ref"):
        ref.domain_read_input()
        ref.parts_read_input(0)
        ref.domain_init.restype = C.c_int
        ref.parts_init.restype = C.c_int
        assert ref.domain_init() == 0
        assert ref.parts_init() == 0
        ref.binDom_init.restype = C.c_int
        assert ref.binDom_init() == 0       # src/bluebottle.c:397-398
    else:
        assert lib.bbb_read_input(b"input") == 0
        assert lib.bbb_domain_init() == 0
        assert lib.bbb_parts_init() == 0
    dom = abi.DomStruct.in_dll(lib, "Dom")
    n = dom.Gcc.s3b
    p = np.ctypeslib.as_array(C.POINTER(C.c_double).in_dll(lib, "p"), shape=(n,))
    if mode.endswith("run"):
        assert lib.bbb_prepare() == 0
        for _ in range(2):
            assert lib.bbb_step() == 0, lib.bbb_status_string(lib.bbb_last_status())
        lib.cuda_dom_pull()
        lib.cuda_part_pull()
    else:
        p[:] = np.sin(np.arange(n) * 0.37)
    snap = {}
    for k, g in FACE.items():
        snap[k] = np.ctypeslib.as_array(C.POINTER(C.c_double).in_dll(lib, k),
                                        shape=(getattr(dom, g).s3b,)).copy()
    for k in CELL:
        snap[k] = np.ctypeslib.as_array(C.POINTER(C.c_double).in_dll(lib, k),
                                        shape=(n,)).copy()
    nparts = C.c_int.in_dll(lib, "nparts").value
    if nparts:
        pp = C.POINTER(abi.PartStruct).in_dll(lib, "parts")
        recs = (abi.PartStruct * nparts).from_address(C.addressof(pp.contents))
        snap["parts_xyz"] = np.array([[q.x, q.y, q.z, q.u, q.v, q.w] for q in recs])
    os.makedirs("output", exist_ok=True)
    C.c_int.in_dll(lib, "rec_paraview_stepnum_out").value = 0
    ref.out_VTK()
    text = open(os.path.join("output", "out_0_0.vtr")).read()
    m = re.search(r'Name="p">\n(.*?)\n</DataArray>', text, re.S)
    snap["vtk_p"] = np.array([float(x) for x in m.group(1).split()])
    g = dom.Gcc
    inner = np.array([p[i + j * g.s1b + k * g.s2b]
                      for k in range(g.ks, g.ke) for j in range(g.js, g.je)
                      for i in range(getattr(g, "is"), g.ie)])
    snap["p_inner"] = inner
    if mode.endswith("run"):
        lib.bbb_release()
    np.savez(out, **snap)


if __name__ == "__main__":
    main()
