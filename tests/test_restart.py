"""The reference's restart file (out_restart src/domain.c:3223, in_restart
:3318): bbb_out_restart / bbb_in_restart against the reference's own writer
and reader, compiled unmodified from its sources into oracle/_ref -- both the
explicit build and the -DIMPLICIT build, whose file omits the diffusion
histories.  Every array, record and scalar of the file is filled with seeded
random values first, so a misplaced or missing run shows up."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from bluebottle_b200 import Sim, abi, configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
from tests.helpers import REF_SRC as REFSRC  # noqa: E402

FACE = {"u": "Gfx", "u0": "Gfx", "diff0_u": "Gfx", "conv0_u": "Gfx",
        "diff_u": "Gfx", "conv_u": "Gfx", "u_star": "Gfx",
        "v": "Gfy", "v0": "Gfy", "diff0_v": "Gfy", "conv0_v": "Gfy",
        "diff_v": "Gfy", "conv_v": "Gfy", "v_star": "Gfy",
        "w": "Gfz", "w0": "Gfz", "diff0_w": "Gfz", "conv0_w": "Gfz",
        "diff_w": "Gfz", "conv_w": "Gfz", "w_star": "Gfz"}
CELL = ("p", "phi", "p0")
INTS = {"phase": "Gcc", "phase_shell": "Gcc", "flag_u": "Gfx",
        "flag_v": "Gfy", "flag_w": "Gfz"}
COEF = ("pnm_re pnm_im pnm_re0 pnm_im0 pnm_re00 pnm_im00 phinm_re phinm_im "
        "phinm_re0 phinm_im0 phinm_re00 phinm_im00 chinm_re chinm_im "
        "chinm_re0 chinm_im0 chinm_re00 chinm_im00").split()
REALS = ("ttime dt0 dt rec_flow_field_ttime_out rec_paraview_ttime_out "
         "rec_particle_ttime_out rec_restart_ttime_out rec_prec_ttime_out "
         "pid_int pid_back").split()
INTS1 = ("stepnum", "rec_paraview_stepnum_out")


def _reflib(implicit):
    if os.path.isdir(REFSRC):
        subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "ref.mk"),
                        "REF=" + REFSRC], check=True, cwd=ROOT)
    path = os.path.join(ROOT, "oracle", "_ref", "libref_host_implicit.so"
                        if implicit else "libref_host.so")
    if not os.path.exists(path):
        pytest.skip("the reference tree is not available to build oracle/_ref")
    return C.CDLL(path, mode=os.RTLD_LOCAL | getattr(os, "RTLD_DEEPBIND", 0))


def _arrays(lib, dom, names, ctype=C.c_double):
    """numpy views of pointer globals of `lib` sized by `dom`'s grids"""
    out = {}
    for name, grid in names.items():
        n = getattr(dom, grid).s3b
        ptr = C.POINTER(ctype).in_dll(lib, name)
        out[name] = np.ctypeslib.as_array(ptr, shape=(n,)) if ptr else None
    return out


def _state(lib, dom, nparts, stride, implicit):
    """every run of the file as numpy views / ctypes objects of `lib`"""
    face = {k: g for k, g in FACE.items() if not (implicit and k.startswith("diff0"))}
    st = _arrays(lib, dom, face)
    st.update(_arrays(lib, dom, {k: "Gcc" for k in CELL}))
    st.update(_arrays(lib, dom, INTS, C.c_int))
    nc = nparts * stride
    for k in COEF:
        st[k] = np.ctypeslib.as_array(C.POINTER(C.c_double).in_dll(lib, k), shape=(nc,))
    pp = C.POINTER(abi.PartStruct).in_dll(lib, "parts")
    st["parts"] = np.ctypeslib.as_array(
        C.cast(pp, C.POINTER(C.c_uint8)), shape=(nparts * C.sizeof(abi.PartStruct),))
    st["bc_plane_pos"] = np.ctypeslib.as_array((C.c_double * 9).in_dll(lib, "bc_plane_pos"))
    return st


def _scalars(lib):
    vals = {k: C.c_double.in_dll(lib, k).value for k in REALS}
    vals.update({k: C.c_int.in_dll(lib, k).value for k in INTS1})
    gp = abi.GStruct.in_dll(lib, "gradP")
    vals["gradP.z"], vals["gradP.zm"] = gp.z, gp.zm
    return vals


def _set_gradp_z(lib, value):
    abi.GStruct.in_dll(lib, "gradP").z = value


@pytest.mark.parametrize("implicit", [0, 1])
def test_restart_file_matches_reference(tmp_path, implicit):
    ref = _reflib(implicit)
    d = tmp_path / "run"
    (d / "input").mkdir(parents=True)
    flow = dict(n=(20, 12, 16), lo=(0.0, 0.0, 0.0), hi=(2.0, 1.2, 1.6), nu=0.05,
                periodic=(True, True, False), pp_residual=1e-9)
    parts = [dict(r=0.2, x=0.5, y=0.6, z=0.8, order=4, rsr=1.2),
             dict(r=0.25, x=1.4, y=0.5, z=0.7, order=4, rsr=1.2)]
    configs.write_flow_config(str(d / "input" / "flow.config"), **flow)
    configs.write_part_config(str(d / "input" / "part.config"), parts)
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
    sim = Sim(input_dir=str(d / "input"), options=dict(implicit=implicit))
    try:
        lib, dom = sim.lib, sim.dom
        nparts, stride = sim.nparts, sim.scalar("coeff_stride")
        assert (nparts, stride) == (2, 15)
        ours = _state(lib, dom, nparts, stride, implicit)
        rng = np.random.default_rng(11)
        for k, a in ours.items():
            if a.dtype == np.float64:
                a[:] = rng.standard_normal(a.size)
            elif a.dtype == np.int32:
                a[:] = rng.integers(-5, 1000, a.size)
            else:
                a[:] = rng.integers(0, 256, a.size)
        for k in REALS:
            C.c_double.in_dll(lib, k).value = float(rng.standard_normal())
        for k in INTS1:
            C.c_int.in_dll(lib, k).value = int(rng.integers(0, 10 ** 6))
        _set_gradp_z(lib, float(rng.standard_normal()))
        want = {k: a.copy() for k, a in ours.items()}
        want_s = _scalars(lib)

        path = str(d / "input" / "restart.config")
        sim.out_restart(path)
        mine = open(path, "rb").read()

        # the reference's reader takes our file into its own globals
        os.chdir(d)
        try:
            ref.in_restart()
        finally:
            os.chdir(cwd)
        theirs = _state(ref, abi.DomStruct.in_dll(ref, "Dom"), nparts, stride, implicit)
        for k in want:
            assert np.array_equal(theirs[k].view(np.uint8), want[k].view(np.uint8)), k
        assert _scalars(ref) == want_s

        # and its writer gives back the same bytes
        os.chdir(d)
        try:
            ref.out_restart()
        finally:
            os.chdir(cwd)
        assert open(path, "rb").read() == mine
        faces = sum(getattr(dom, g).s3b for g in ("Gfx", "Gfy", "Gfz"))
        cc = dom.Gcc.s3b
        size = (3 * 8 + 2 * 4                       # clocks, step counters
                + (6 if implicit else 7) * 8 * faces  # velocity runs
                + 3 * 8 * cc + 2 * 4 * cc + 4 * faces  # p, phi, p0; phase; flags
                + 9 * 8                              # bc_plane_pos
                + nparts * C.sizeof(abi.PartStruct) + 4
                + 18 * 8 * nparts * stride
                + 7 * 8 + 2 * 8)                     # recorder, PID, gradP.z/zm
        assert len(mine) == size

        # our reader restores everything from the reference's file
        for k, a in ours.items():
            a[:] = 0
        for k in REALS:
            C.c_double.in_dll(lib, k).value = 0.
        for k in INTS1:
            C.c_int.in_dll(lib, k).value = 0
        _set_gradp_z(lib, 0.)
        sim.in_restart(path)
        for k in want:
            assert np.array_equal(ours[k].view(np.uint8), want[k].view(np.uint8)), k
        assert _scalars(lib) == want_s
    finally:
        sim.close()


def test_in_restart_rejects_short_file(tmp_path):
    wl = configs.taylor_green(8)
    sim = Sim(wl)
    try:
        path = str(tmp_path / "restart.config")
        sim.out_restart(path)
        data = open(path, "rb").read()
        open(path, "wb").write(data[:len(data) // 2])
        with pytest.raises(Exception):
            sim.in_restart(path)
        assert sim.lib.bbb_last_status() == 3        # BBB_ERR_CONFIG
    finally:
        sim.close()
