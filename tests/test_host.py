"""Host-side logic of the library without a GPU: the reference's input
readers (src/domain.c:30-730, src/particle.c:79-159), the derived domain
set-up, the seeded sphere pack and the gravity balance."""
import math
import os

import numpy as np
import pytest

from bluebottle_b200 import Sim, configs, abi


def _dir_sim(tmp_path, parts, **flow):
    d = str(tmp_path)
    configs.write_flow_config(os.path.join(d, "flow.config"), **flow)
    configs.write_part_config(os.path.join(d, "part.config"), parts)
    return Sim(input_dir=d)


def test_flow_and_part_config_round_trip(tmp_path):
    sim = _dir_sim(tmp_path,
                   [dict(r=0.5, x=0.25, y=0.5, z=0.75, rho=3.0, order=3, rsr=1.3),
                    dict(r=0.4, x=1.0, y=0.2, z=0.4)],
                   n=(12, 10, 8), lo=(-0.6, 0.0, 0.0), hi=(0.6, 1.0, 0.8),
                   nu=0.25, rho_f=2.0, pp_residual=1e-9, pp_max_iter=321,
                   lamb_max_iter=7, lamb_residual=1e-3, lamb_relax=0.9,
                   lamb_cut=1e-5, periodic=(True, False, True),
                   gradP=(0.1, -0.2, 0.3), g=(0.0, 0.0, -9.8))
    d = sim.dom
    assert (d.xn, d.yn, d.zn) == (12, 10, 8)
    assert math.isclose(d.dx, 0.1) and math.isclose(d.dy, 0.1) and math.isclose(d.dz, 0.1)
    assert math.isclose(d.xs, -0.6) and math.isclose(d.xe, 0.6)
    # ghosted grids: one ghost layer, Gfx one face more along x
    assert d.Gcc.inb == 14 and d.Gfx.inb == 15 and d.Gfy.jnb == 13 and d.Gfz.knb == 11
    assert d.Gcc.s1b == d.Gcc.inb and d.Gcc.s2b == d.Gcc.inb * d.Gcc.jnb
    assert sim.scalar("nu") == 0.25 and sim.scalar("rho_f") == 2.0
    assert math.isclose(sim.scalar("mu"), 0.5)
    assert sim.scalar("pp_residual") == 1e-9 and sim.scalar("pp_max_iter") == 321
    assert sim.scalar("lamb_max_iter") == 7
    assert sim.scalar("lamb_relax") == 0.9 and sim.scalar("lamb_cut") == 1e-5
    bc = sim.bc
    assert bc.pW == 0 and bc.pE == 0 and bc.pB == 0          # PERIODIC
    assert bc.pS == 2 and bc.pN == 2                          # NEUMANN
    assert bc.uS == 1 and bc.vN == 1 and bc.wS == 1           # DIRICHLET
    assert sim.gradP.xm == 0.1 and sim.gradP.ym == -0.2 and sim.gradP.zm == 0.3
    assert sim.g.zm == -9.8
    assert sim.nparts == 2
    p = sim.parts()
    assert (p[0].r, p[0].x, p[0].y, p[0].z, p[0].rho, p[0].order) == (0.5, 0.25, 0.5, 0.75, 3.0, 3)
    assert math.isclose(p[1].r, 0.4)
    # coefficient storage: the largest order sets the stride,
    # (order+1)(order+2)/2 modes (src/particle.c)
    assert sim.scalar("coeff_stride") == (3 + 1) * (3 + 2) // 2 or \
        sim.scalar("coeff_stride") == (4 + 1) * (4 + 2) // 2
    sim.close()


def _pair_gaps(x, L):
    d = x[:, None, :] - x[None, :, :]
    d -= L * np.round(d / L)
    r = np.sqrt((d ** 2).sum(-1))
    r[np.diag_indices(len(x))] = np.inf
    return r


def test_seeded_pack_reproducible_and_gapped():
    wl = configs.sedimentation((32, 32, 32), (16.0, 16.0, 16.0), 60, seed=9)
    sims = []
    pos = []
    for _ in range(2):
        s = Sim(wl)
        pos.append(np.array([(q.x, q.y, q.z) for q in s.parts()]))
        L = np.array([s.dom.xl, s.dom.yl, s.dom.zl])
        s.close()
    assert pos[0].shape == (60, 3)
    assert np.array_equal(pos[0], pos[1])
    r = _pair_gaps(pos[0], L)
    assert r.min() >= 2.0 + 0.1 - 1e-12          # surface gap >= 0.1 a
    assert np.all(pos[0] >= 0) and np.all(pos[0] < L)
    other = Sim(configs.sedimentation((32, 32, 32), (16.0, 16.0, 16.0), 60, seed=10))
    p2 = np.array([(q.x, q.y, q.z) for q in other.parts()])
    other.close()
    assert not np.array_equal(pos[0], p2)


def test_gravity_balance_sets_mean_excess_weight():
    wl = configs.sedimentation((32, 32, 32), (16.0, 16.0, 16.0), 20, seed=2)
    s = Sim(wl)
    vol = 4.0 / 3.0 * math.pi
    expect = 20 * (2.0 - 1.0) * vol * (-1.0) / 16.0 ** 3
    assert math.isclose(s.gradP.zm, expect, rel_tol=1e-12)
    s.close()


def test_too_dense_pack_reports_config_error():
    wl = configs.sedimentation((16, 16, 16), (4.0, 4.0, 4.0), 50, seed=1)
    with pytest.raises(Exception):
        Sim(wl)


def test_options_round_trip():
    import ctypes as C
    lib = abi.load()
    o = abi.Options()
    lib.bbb_default_options(C.byref(o))
    assert o.implicit == 1 and o.precision == 0
    o.precision = 1
    o.inner_tol = 3e-6
    lib.bbb_set_options(C.byref(o))
    g = abi.Options()
    lib.bbb_get_options(C.byref(g))
    assert g.precision == 1 and g.inner_tol == 3e-6
    lib.bbb_default_options(C.byref(o))
    lib.bbb_set_options(C.byref(o))


def test_learned_guess_cost_gate():
    """bbb_learn_gate_decide: the saving of a guess whose residual is a
    factor f below the extrapolation's, in a solve that reduced its
    residual by a factor F in t ms, is t ln f / ln F; the evaluation is
    skipped for 8, 16, .. 256 steps while that stays below its cost."""
    import ctypes as C
    lib = abi.load()
    fails, ben = C.c_int(0), C.c_double(0.)

    def decide(cost, t, r_ext, r_start, r_final):
        return lib.bbb_learn_gate_decide(cost, t, r_ext, r_start, r_final,
                                         C.byref(fails), C.byref(ben))

    # a 10x better start of a solve that removes 1e8 in 100 ms saves 12.5 ms
    assert decide(10.0, 100.0, 1.0, 0.1, 1e-9) == 0
    assert math.isclose(ben.value, 100.0 / 8.0) and fails.value == 0
    # a 1.3x better start saves ~1.4 ms: skipped 8, then 16, .. up to 256 steps
    skips = [decide(10.0, 100.0, 1.3, 1.0, 1e-8) for _ in range(8)]
    assert skips == [8, 16, 32, 64, 128, 256, 256, 256]
    assert math.isclose(ben.value, 100.0 * math.log(1.3) / math.log(1e8))
    # a guess that was not used saves nothing; a paying one resets the count
    assert decide(0.1, 100.0, 1.0, 1.0, 1e-8) == 256 and ben.value == 0.0
    assert decide(1.0, 100.0, 1.0, 0.01, 1e-8) == 0 and fails.value == 0
    # degenerate solves (already converged, no time) save nothing
    assert decide(0.0, 100.0, 1.0, 1e-9, 1e-8) == 8 and ben.value == 0.0
    assert decide(0.0, 0.0, 1.0, 0.1, 1e-8) == 16


def test_learned_guess_crops_per_step_range():
    """bbb_learn_set_crops_per_step takes 1..64 crops per recorded solve and
    refuses anything else with BBB_ERR_CONFIG, keeping the setting it had
    (no device is touched)."""
    lib = abi.load()
    ERR_CONFIG = 3
    lib.bbb_clear_status()
    for bad in (0, -1, 65, 1000):
        assert lib.bbb_learn_set_crops_per_step(bad) == ERR_CONFIG
    for good in (1, 32, 64):
        assert lib.bbb_learn_set_crops_per_step(good) == 0
    assert lib.bbb_learn_set_crops_per_step(8) == 0
    assert lib.bbb_last_status() == 0


def _walled_sim(tmp_path, periodic, screens=(0.0, 0.0)):
    """a 16 x 16 x 12 box without particles; non-periodic axes are walls,
    the bottom/top screens (bc.dsB, bc.dsT) as given"""
    d = str(tmp_path)
    os.makedirs(d, exist_ok=True)
    configs.write_flow_config(os.path.join(d, "flow.config"), n=(32, 32, 24),
                              hi=(16.0, 16.0, 12.0), periodic=periodic)
    configs.write_part_config(os.path.join(d, "part.config"), [])
    sim = Sim(input_dir=d)
    b = abi.BCStruct.in_dll(sim.lib, "bc")
    b.dsB, b.dsT = screens
    return sim


def test_seeded_pack_respects_walls_screens_and_periodic_axes(tmp_path):
    """The reference seeder's placement rules (src/seeder.c:246-700): centres
    inside the screened domain, a (+ half the gap) from its non-periodic
    walls, the gap counted through periodic images only along periodic
    axes."""
    sim = _walled_sim(tmp_path, (True, True, False), screens=(1.0, 2.0))
    try:
        lib = sim.lib
        assert lib.bbb_seed_particles(120, 1.0, 0.2, 2.0, 4, 1.2, 5) == 0
        pos = np.array([(q.x, q.y, q.z) for q in sim.parts()])
        assert pos.shape == (120, 3)
        wall = 1.0 + 0.1
        assert pos[:, 2].min() >= 0.0 + 1.0 + wall - 1e-12
        assert pos[:, 2].max() <= 12.0 - 2.0 - wall + 1e-12
        assert np.all(pos[:, :2] >= 0) and np.all(pos[:, :2] < 16.0)
        dd = pos[:, None, :] - pos[None, :, :]
        dd[..., :2] -= 16.0 * np.round(dd[..., :2] / 16.0)   # x, y periodic
        r = np.sqrt((dd ** 2).sum(-1)) + np.eye(len(pos)) * 1e9
        assert r.min() >= 2.0 + 0.2 - 1e-12
        # no room: centres 1.1 from both screened faces of a 2-wide slab
        b = abi.BCStruct.in_dll(lib, "bc")
        b.dsB, b.dsT = 5.0, 5.0
        assert lib.bbb_seed_particles(1, 1.0, 0.2, 2.0, 4, 1.2, 5) == 3
    finally:
        sim.close()


def test_pack_reproducible_with_walls(tmp_path):
    pos = []
    for k in range(2):
        sim = _walled_sim(tmp_path / str(k), (False, True, False))
        try:
            assert sim.lib.bbb_seed_particles(80, 1.0, 0.1, 2.0, 4, 1.2, 11) == 0
            pos.append(np.array([(q.x, q.y, q.z) for q in sim.parts()]))
        finally:
            sim.close()
    assert np.array_equal(pos[0], pos[1])
    assert pos[0][:, 0].min() >= 1.05 - 1e-12 and pos[0][:, 0].max() <= 16.0 - 1.05 + 1e-12


def test_written_part_config_reads_back(tmp_path):
    """bbb_write_part_config writes the reference's part.config layout; the
    library's reader (the restatement of src/particle.c:79) and, when the
    reference tree is here, the reference's own parts_read_input read it
    back to the same doubles."""
    wl = configs.sedimentation((32, 32, 32), (16.0, 16.0, 16.0), 25, seed=4)
    sim = Sim(wl)
    run = tmp_path / "run"
    (run / "input").mkdir(parents=True)
    try:
        sim.set_scalar("interactionLengthRatio", 0.375)
        want = [(q.r, q.x, q.y, q.z, q.rho, q.E, q.sigma, q.e_dry, q.coeff_fric,
                 q.order, q.rs, q.translating, q.rotating) for q in sim.parts()]
        sim.write_part_config(str(run / "input" / "part.config"))
        configs.write_flow_config(str(run / "input" / "flow.config"), n=(32, 32, 32),
                                  hi=(16.0, 16.0, 16.0))
    finally:
        sim.close()
    text = open(run / "input" / "part.config").read()
    assert text.startswith("n 25\n(l/a) 0.375\n\nr 1\n(x, y, z) ")
    back = Sim(input_dir=str(run / "input"))
    try:
        got = [(q.r, q.x, q.y, q.z, q.rho, q.E, q.sigma, q.e_dry, q.coeff_fric,
                q.order, q.rs, q.translating, q.rotating) for q in back.parts()]
        assert got == want
        assert back.scalar("interactionLengthRatio") == 0.375
    finally:
        back.close()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    from tests.helpers import REF_SRC
    if os.path.isdir(REF_SRC):
        import subprocess
        subprocess.run(["make", "-s", "-f", os.path.join(root, "oracle", "ref.mk"),
                        "REF=" + REF_SRC], check=True, cwd=root)
    ref = os.path.join(root, "oracle", "_ref", "libref_host.so")
    if not os.path.exists(ref):
        return
    import ctypes as C
    lib = C.CDLL(ref, mode=os.RTLD_LOCAL | getattr(os, "RTLD_DEEPBIND", 0))
    cwd = os.getcwd()
    os.chdir(run)
    try:
        lib.parts_read_input(0)
    finally:
        os.chdir(cwd)
    assert C.c_int.in_dll(lib, "nparts").value == 25
    assert C.c_double.in_dll(lib, "interactionLengthRatio").value == 0.375
    pp = C.POINTER(abi.PartStruct).in_dll(lib, "parts")
    for i, w in enumerate(want):
        q = pp[i]
        assert (q.r, q.x, q.y, q.z, q.rho, q.E, q.sigma, q.e_dry, q.coeff_fric,
                q.order, q.rs, q.translating, q.rotating) == w
