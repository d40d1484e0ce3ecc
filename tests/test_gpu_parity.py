"""GPU (libbbb200.so through its C ABI) against the FP64 CPU oracle on the
same seeded inputs.  Integer arrays (phase, phase_shell, flags) must match
bit for bit; floating-point fields within the tolerances stated per test."""
import numpy as np
import pytest

from bluebottle_b200 import Sim, configs
from oracle.orc import Oracle
from tests.helpers import rel_err, field_interior

pytestmark = pytest.mark.gpu

# both sides solve to the same relative residual from the same iterate; the
# difference is summation order only
FIELD_TOL = 1e-9
# the pressure correction phi is the Poisson solution itself: two solves
# stopped at ||r|| <= tol ||b|| may differ by up to cond(A) * tol relative
# (here tol = 1e-10 and cond ~ 1e3 on 32^3)
PHI_TOL = 1e-7


def _run_pair(wl, steps, options=None):
    sim = Sim(wl, options=options)
    orc = Oracle.from_sim(sim)
    sim.prepare()
    out = []
    for _ in range(steps):
        sim.step()
        orc.step()
        sim.pull()
        out.append((sim.stats(), orc.stats()))
    return sim, orc, out


def test_taylor_green_steps(gpu):
    wl = configs.taylor_green(32)
    sim, orc, stats = _run_pair(wl, 3)
    try:
        d = sim.dom
        for name in ("u", "v", "w", "p", "phi"):
            e = rel_err(field_interior(d, name, sim.array(name)),
                        field_interior(d, name, orc.field(name)))
            assert e < (PHI_TOL if name == "phi" else FIELD_TOL), (name, e)
        # the GPU takes rho' for beta as (rh, s) - omega (rh, t) (one pass
        # fewer per iteration); iterates follow CUSP's to rounding, and the
        # iteration count of a smooth right-hand side moves by a few under
        # rounding alone (either recurrence, FP64): the oracle's own count
        # at the third step ranged 22-26 over the summation orders of 1-8
        # OpenMP threads before its dot products were given a fixed order
        for g, c in stats:
            assert abs(g.pp_iters_last - c["pp_iters"]) <= max(4, 0.15 * c["pp_iters"])
        e_gpu, e_orc = sim.energy(), orc.energy()
        assert abs(e_gpu - e_orc) / e_orc < 1e-11
    finally:
        sim.close()
        orc.close()


@pytest.mark.parametrize("reliable", [0, 1])
def test_mixed_precision_matches_fp64_oracle(gpu, reliable):
    """FP32 inner solves inside FP64 defect correction reach the same FP64
    residual test; fields agree with the FP64 oracle to within what that
    tolerance allows (cond * tol, here < 1e-7).  With reliable updates the
    single-mode Taylor-Green residual makes every resumed sweep break down
    (the shadow residual is the mode, the replaced residual rounding noise):
    the sweep falls back to a restart and the solve still converges."""
    wl = configs.taylor_green(32)
    sim, orc, stats = _run_pair(wl, 3, options=dict(precision=1,
                                                     inner_tol=1e-4,
                                                     reliable=reliable))
    try:
        d = sim.dom
        for name in ("u", "v", "w", "p"):
            e = rel_err(field_interior(d, name, sim.array(name)),
                        field_interior(d, name, orc.field(name)))
            assert e < 1e-7, (name, e)
        for g, _ in stats:
            assert g.pp_resid_last <= 1e-10
            assert g.pp_outer_last >= 1
    finally:
        sim.close()
        orc.close()


def test_explicit_ab2_steps(gpu):
    wl = configs.taylor_green(32)
    wl.options["implicit"] = 0
    sim, orc, _ = _run_pair(wl, 2)
    try:
        d = sim.dom
        for name in ("u", "v", "w", "p"):
            e = rel_err(field_interior(d, name, sim.array(name)),
                        field_interior(d, name, orc.field(name)))
            assert e < FIELD_TOL, (name, e)
    finally:
        sim.close()
        orc.close()


def _small_particle_case(npart=4, n=32, side=8.0, seed=3):
    wl = configs.sedimentation((n, n, n), (side, side, side), npart, nu=0.1,
                               tol=1e-10, lamb_max_iter=4, seed=seed)
    return wl


def test_cage_integer_parity(gpu):
    wl = _small_particle_case(npart=6)
    sim = Sim(wl)
    orc = Oracle.from_sim(sim)
    sim.prepare()
    sim.pull()
    try:
        for name in ("phase", "phase_shell", "flag_u", "flag_v", "flag_w"):
            a, b = sim.array(name), orc.field(name)
            assert np.array_equal(a, b), (name, int(np.sum(a != b)))
        assert int(np.sum(sim.array("phase") > -1)) > 0
        for pg, po in zip(sim.parts(), orc.field("parts")):
            for k in ("is", "ibs", "ie", "ibe", "js", "jbs", "je", "jbe",
                      "ks", "kbs", "ke", "kbe", "in", "jn", "kn", "cx", "cy",
                      "cz"):
                assert getattr(pg.cage, k) == getattr(po.cage, k), k
    finally:
        sim.close()
        orc.close()


def test_particle_step_parity(gpu):
    wl = _small_particle_case(npart=4)
    sim, orc, stats = _run_pair(wl, 2)
    try:
        d = sim.dom
        for name in ("phase", "flag_u", "flag_v", "flag_w"):
            assert np.array_equal(sim.array(name), orc.field(name)), name
        for name in ("u", "v", "w", "p"):
            e = rel_err(field_interior(d, name, sim.array(name)),
                        field_interior(d, name, orc.field(name)))
            assert e < 1e-7, (name, e)
        for name in ("pnm_re", "phinm_re", "chinm_re"):
            e = rel_err(sim.array(name), orc.field(name))
            assert e < 1e-7, (name, e)
        for pg, po in zip(sim.parts(), orc.field("parts")):
            for k in ("x", "y", "z", "u", "v", "w", "Fx", "Fy", "Fz"):
                a, b = getattr(pg, k), getattr(po, k)
                assert abs(a - b) <= 1e-7 * max(1.0, abs(b)), (k, a, b)
        for g, c in stats:
            assert g.lamb_iters == c["lamb_iters"]
    finally:
        sim.close()
        orc.close()


@pytest.mark.parametrize("reliable,itol", [(0, 1e-4), (1, 1e-2)])
def test_mixed_precision_vector_paths_with_particles(gpu, reliable, itol):
    """FP32-inner form on a 128-cell row length, so the tensor-map staged
    FP32 BiCGSTAB passes and the 2-wide FP64 stencil paths run (Poisson and
    the v, w Helmholtz systems; u has 129 faces per row and takes the scalar
    path), with spheres: fields within what the 1e-10 stopping rule allows
    of the FP64 oracle, with restarted and with resumed (reliable-update)
    inner sweeps."""
    wl = configs.sedimentation((128, 32, 32), (32.0, 8.0, 8.0), 4, nu=0.1,
                               tol=1e-10, lamb_max_iter=2, seed=5, prec=1)
    sim, orc, stats = _run_pair(wl, 2, options=dict(precision=1,
                                                     lamb_max_iter_override=2,
                                                     reliable=reliable,
                                                     inner_tol=itol))
    try:
        d = sim.dom
        for name in ("u", "v", "w", "p"):
            e = rel_err(field_interior(d, name, sim.array(name)),
                        field_interior(d, name, orc.field(name)))
            assert e < 1e-7, (name, e)
        for g, _ in stats:
            assert g.pp_resid_last <= 1e-10
            assert g.helm_iters_total > 0
        for pg, po in zip(sim.parts(), orc.field("parts")):
            for k in ("x", "z", "u", "w", "Fz"):
                a, b = getattr(pg, k), getattr(po, k)
                assert abs(a - b) <= 1e-7 * max(1.0, abs(b)), (k, a, b)
    finally:
        sim.close()
        orc.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_u_system_stored_y_fastest(gpu, precision):
    """33 faces per x row but 128 cells per y row: the u Crank-Nicolson
    system is stored y-fastest (so its passes take the 4-wide FP32 / 2-wide
    FP64 kernels and the staged outer residual), the v, w systems and the
    Poisson system x-fastest; fields and spheres within what the 1e-10
    stopping rule allows of the FP64 oracle, in both precision forms."""
    wl = configs.sedimentation((32, 128, 32), (8.0, 32.0, 8.0), 4, nu=0.1,
                               tol=1e-10, lamb_max_iter=2, seed=9, prec=precision)
    sim, orc, stats = _run_pair(wl, 2, options=dict(precision=precision,
                                                     lamb_max_iter_override=2))
    try:
        d = sim.dom
        for name in ("u", "v", "w", "p"):
            e = rel_err(field_interior(d, name, sim.array(name)),
                        field_interior(d, name, orc.field(name)))
            assert e < 1e-7, (name, e)
        for g, _ in stats:
            assert g.helm_iters_total > 0
        for pg, po in zip(sim.parts(), orc.field("parts")):
            for k in ("x", "z", "u", "w", "Fz"):
                a, b = getattr(pg, k), getattr(po, k)
                assert abs(a - b) <= 1e-7 * max(1.0, abs(b)), (k, a, b)
    finally:
        sim.close()
        orc.close()


def test_pid_controller_parity(gpu):
    """The reference's PID control of the driving pressure gradient
    (src/cuda_bluebottle.cu:3781-3805: gradP.z follows the spheres' mean
    vertical acceleration with gains Kp, Ki, Kd, computed on the host from
    the pulled particle records).  With nonzero gains the library and the
    FP64 oracle step together and agree on gradP.z, the controller's
    integral and last input, the fields and the spheres."""
    import ctypes as C
    wl = configs.sedimentation((32, 32, 64), (8.0, 8.0, 16.0), 4, nu=0.1,
                               tol=1e-10, lamb_max_iter=2, seed=6)
    sim = Sim(wl, options=dict(lamb_max_iter_override=2))
    gains = (("Kp", 0.5), ("Ki", 0.1), ("Kd", 0.05))
    for nm, v in gains:
        C.c_double.in_dll(sim.lib, nm).value = v
    try:
        orc = Oracle.from_sim(sim)
    except BaseException:
        sim.close()
        raise
    try:
        assert orc.P.Kp == 0.5 and orc.P.Ki == 0.1 and orc.P.Kd == 0.05
        sim.prepare()
        gz0 = sim.gradP.z
        for _ in range(3):
            sim.step()
            orc.step()
            a, b = sim.gradP.z, orc.P.gradP.z
            assert abs(a - b) <= 1e-9 * max(abs(b), 1e-12), (a, b)
            for nm in ("pid_int", "pid_back"):
                x = C.c_double.in_dll(sim.lib, nm).value
                y = getattr(orc.P, nm)
                assert abs(x - y) <= 1e-9 * max(abs(y), 1e-12), (nm, x, y)
        assert sim.gradP.z != gz0          # the controller acted
        sim.pull()
        d = sim.dom
        for name in ("u", "v", "w", "p"):
            e = rel_err(field_interior(d, name, sim.array(name)),
                        field_interior(d, name, orc.field(name)))
            assert e < 1e-8, (name, e)
        for pg, po in zip(sim.parts(), orc.field("parts")):
            for k in ("z", "w", "wdot"):
                a, b = getattr(pg, k), getattr(po, k)
                assert abs(a - b) <= 1e-8 * max(1.0, abs(b)), (k, a, b)
    finally:
        sim.close()
        orc.close()
