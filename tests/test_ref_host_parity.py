"""The library's host set-up against the reference's own code.

oracle/ref.mk compiles the reference's src/domain.c, src/particle.c and
src/rng.c unmodified into oracle/_ref/libref_host.so.  Both read the same
flow.config / part.config; the domain structs, boundary conditions, scalar
globals, particle records and initial fields must then be identical, field
for field (domain_read_input src/domain.c:30, domain_init :1591,
parts_read_input src/particle.c:79, parts_init :295, binDom_init :598).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from bluebottle_b200 import Sim, abi, configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFLIB = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
from tests.helpers import REF_SRC as REFSRC  # noqa: E402


def _reflib():
    if os.path.isdir(REFSRC):
        subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "ref.mk"),
                        "REF=" + REFSRC], check=True, cwd=ROOT)
    if not os.path.exists(REFLIB):
        pytest.skip("the reference tree is not available to build oracle/_ref")
    return C.CDLL(REFLIB, mode=os.RTLD_LOCAL | getattr(os, "RTLD_DEEPBIND", 0))


REAL_SCALARS = ("dt", "dt0", "ttime", "rho_f", "nu", "mu", "CFL", "pp_residual",
                "lamb_residual", "lamb_relax", "lamb_cut", "vel_tDelay",
                "p_tDelay", "g_tDelay", "duration", "Kp", "Ki", "Kd")
INT_SCALARS = ("pp_max_iter", "lamb_max_iter", "out_plane", "init_cond",
               "nparts", "coeff_stride", "stepnum")
FIELDS = (("p0", "Gcc"), ("p", "Gcc"), ("phi", "Gcc"), ("u", "Gfx"),
          ("u0", "Gfx"), ("v", "Gfy"), ("v0", "Gfy"), ("w", "Gfz"),
          ("w0", "Gfz"), ("conv0_u", "Gfx"), ("diff0_w", "Gfz"))


def _run_reference(ref, d):
    cwd = os.getcwd()
    os.chdir(d)
    try:
        ref.domain_read_input()
        ref.parts_read_input(0)
        ref.domain_init.restype = C.c_int
        ref.parts_init.restype = C.c_int
        assert ref.domain_init() == 0
        assert ref.parts_init() == 0
    finally:
        os.chdir(cwd)


def _diff(a, b, path=""):
    """Named fields that differ (padding bytes are not compared)."""
    out = []
    if isinstance(a, C.Structure):
        for f, _ in a._fields_:
            out += _diff(getattr(a, f), getattr(b, f), path + "." + f)
    elif isinstance(a, C.Array):
        for i in range(len(a)):
            out += _diff(a[i], b[i], "%s[%d]" % (path, i))
    elif a != b:
        out.append((path, a, b))
    return out


@pytest.mark.parametrize("case", ["periodic", "walls_shear", "channel_parts"])
def test_host_setup_matches_reference(tmp_path, case):
    ref = _reflib()
    d = tmp_path / "run"
    (d / "input").mkdir(parents=True)
    flow = dict(n=(24, 20, 16), lo=(-1.2, 0.0, 0.5), hi=(1.2, 2.0, 2.1),
                nu=0.07, rho_f=1.3, pp_residual=1e-9, pp_max_iter=777,
                lamb_max_iter=5, lamb_residual=2e-3, lamb_relax=0.8,
                lamb_cut=3e-5, gradP=(0.01, 0.0, -0.2), g=(0.0, -0.5, -1.0))
    parts = []
    if case == "walls_shear":
        flow.update(periodic=(True, False, False), init_cond="SHEAR")
    elif case == "channel_parts":
        flow.update(periodic=(True, True, False), init_cond="CHANNEL")
        parts = [dict(r=0.3, x=0.1, y=0.5, z=1.0, rho=2.5, order=4, rsr=1.2),
                 dict(r=0.25, x=-0.6, y=1.4, z=1.6, rho=1.1, order=3, rsr=1.3,
                      translating=0, rotating=1)]
    configs.write_flow_config(str(d / "input" / "flow.config"), **flow)
    configs.write_part_config(str(d / "input" / "part.config"), parts)
    _run_reference(ref, str(d))
    sim = Sim(input_dir=str(d / "input"))
    try:
        lib = sim.lib
        assert _diff(abi.DomStruct.in_dll(ref, "Dom"), sim.dom, "Dom") == []
        rd = C.POINTER(abi.DomStruct).in_dll(ref, "dom").contents
        md = C.POINTER(abi.DomStruct).in_dll(lib, "dom").contents
        assert _diff(rd, md, "dom[0]") == []
        assert _diff(abi.BCStruct.in_dll(ref, "bc"), sim.bc, "bc") == []
        ref.binDom_init.restype = C.c_int
        assert ref.binDom_init() == 0
        assert _diff(abi.DomStruct.in_dll(ref, "binDom"),
                     abi.DomStruct.in_dll(lib, "binDom"), "binDom") == []
        for g in ("g", "gradP"):
            assert _diff(abi.GStruct.in_dll(ref, g), abi.GStruct.in_dll(lib, g), g) == []
        for s in REAL_SCALARS:
            assert C.c_double.in_dll(ref, s).value == sim.scalar(s), s
        for s in INT_SCALARS:
            assert C.c_int.in_dll(ref, s).value == sim.scalar(s), s
        dom = sim.dom
        for name, grid in FIELDS:
            n = getattr(dom, grid).s3b
            a = np.ctypeslib.as_array(C.POINTER(C.c_double).in_dll(ref, name), shape=(n,))
            assert np.array_equal(a, sim.array(name)), name
        n = sim.nparts
        assert n == len(parts)
        if n:
            rp = (abi.PartStruct * n).from_address(
                C.addressof(C.POINTER(abi.PartStruct).in_dll(ref, "parts").contents))
            mp = sim.parts()
            for q in range(n):
                # `bin` is left uninitialised by the reference's malloc until
                # the collision binning fills it (src/bluebottle_kernel.cu:2437)
                d = [x for x in _diff(rp[q], mp[q], "parts[%d]" % q)
                     if not x[0].endswith(".bin")]
                assert d == [], d
    finally:
        sim.close()


def test_reference_arm_setup_matches_library(tmp_path):
    """The benchmark's reference arm sets up through the reference's own
    readers and initialisation (oracle/_ref/libref_host_implicit.so) from
    the seeded inputs oracle/seed.py writes; that state, copied into the
    oracle, equals the state the library's own set-up gives the oracle."""
    from oracle.orc import Oracle, reference_host_lib, reference_setup
    from oracle.seed import write_workload_inputs
    if os.path.isdir(REFSRC):
        subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "ref.mk"),
                        "REF=" + REFSRC], check=True, cwd=ROOT)
    if reference_host_lib(True) is None:
        pytest.skip("the reference tree is not available to build oracle/_ref")
    wl = configs.sedimentation((32, 32, 32), (8.0, 8.0, 8.0), 6, nu=0.05,
                               gap=0.5, loa=1.0, seed=5)
    run = tmp_path / "run"
    write_workload_inputs(wl, str(run / "input"))
    ref = reference_setup(str(run), implicit=True)
    a = Oracle.from_reference(ref, implicit=1, lamb_override=3, prepare=False)
    sim = Sim(wl, options=dict(lamb_max_iter_override=3))
    try:
        b = Oracle.from_sim(sim, prepare=False)
    finally:
        sim.close()
    try:
        assert _diff(a.dom, b.dom, "dom") == []
        pa, pb = a.P, b.P
        d = [x for x in _diff(pa, pb, "P")]
        assert d == [], d
        for name in Oracle.FIELD_NAMES:
            assert np.array_equal(a.field(name), b.field(name)), name
        ra, rb = a.field("parts"), b.field("parts")
        assert len(ra) == len(rb) == 6
        for q in range(6):
            d = [x for x in _diff(ra[q], rb[q], "parts[%d]" % q)
                 if not x[0].endswith(".bin")]
            assert d == [], d
    finally:
        a.close()
        b.close()
