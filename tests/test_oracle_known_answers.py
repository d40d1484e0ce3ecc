"""The oracle against closed-form answers, on the CPU.

The reference ships no stored golden outputs; its in-binary harness
(src/cuda_testing.cu) checks analytic fields.  These tests turn those cases
into assertions on the oracle: the Stokes sphere of cuda_lamb_test
(src/cuda_testing.cu:1836-2230), the boundary ghosts of cuda_BC_test
(:547, kernels src/bluebottle_kernel.cu:26-1248), the projection of
cuda_project_test (:1250), plus the Taylor-Green viscous decay and a
manufactured Poisson solution.
"""
import math
import os

import numpy as np
import pytest

from bluebottle_b200 import Sim, configs
from oracle.orc import Oracle

from tests.helpers import stokes_case, stokes_fields


# ---------------------------------------------------------------- Stokes
def test_stokes_sphere_drag_and_lamb_boundary_values(tmp_path):
    """Uniform Stokes flow W past a sphere of radius a at the origin (mu = 1):
    the Lamb quadrature must recover the Stokes drag 6 pi mu a W along z,
    no side force or torque, and part_BC must reproduce the analytic
    velocity on the faces it sets."""
    W, a, mu = 0.01, 1.0, 1.0
    sim = stokes_case(tmp_path, n=48, L=3.0)
    fields = stokes_fields(sim, W=W, a=a)
    for nm, arr in fields.items():
        sim.array(nm)[:] = arr
    o = Oracle.from_sim(sim, prepare=False)
    sim.close()
    o.lib.orc_build_cages(o.st)
    o.lib.orc_Lamb(o.st)
    pt = o.field("parts")[0]
    drag = 6.0 * math.pi * mu * a * W
    assert abs(pt.Fz - drag) / drag < 2e-3
    assert abs(pt.Fx) < 1e-12 and abs(pt.Fy) < 1e-12
    assert max(abs(pt.Lx), abs(pt.Ly), abs(pt.Lz)) < 1e-9
    o.lib.orc_part_BC(o.st, 0)
    for nm in ("u", "v", "w"):
        got = o.field(nm)
        flag = o.field("flag_" + nm)
        set_ = got != fields[nm]
        assert set_.sum() > 100                     # faces near the sphere
        assert np.all(flag[set_] < 1)
        err = np.abs(got - fields[nm])[set_].max()
        assert err < 3e-5, (nm, err)                # 0.3% of W
    o.close()


# ---------------------------------------------------------------- TG decay
def test_taylor_green_decay_matches_discrete_eigenvalue():
    """3-D Taylor-Green, 32^3, nu = 0.01, dt = 0.01: at early times the
    kinetic energy decays as exp(-2 nu lambda t) with lambda the discrete
    Laplacian eigenvalue of the mode, 3 (2/dx sin(dx/2))^2."""
    sim = Sim(configs.taylor_green(32))
    o = Oracle.from_sim(sim, prepare=True)
    sim.close()
    E0 = o.energy()
    steps = 10
    for _ in range(steps):
        assert o.step() == 0
    E = o.energy()
    dx = 2 * math.pi / 32
    lam = 3.0 * (2.0 / dx * math.sin(dx / 2)) ** 2
    expect = math.exp(-2 * 0.01 * lam * steps * 0.01)
    assert abs(E / E0 - expect) < 2e-5
    mx, _ = o.divergence()
    assert mx < 1e-10
    o.close()


# ---------------------------------------------------------------- Poisson
def test_poisson_manufactured_solution():
    """A x = b for a random zero-mean x on the periodic 24^3 operator: the
    Jacobi-BiCGSTAB restatement recovers x to the solver tolerance."""
    import ctypes as C
    sim = Sim(configs.taylor_green(24))
    o = Oracle.from_sim(sim, prepare=False)
    sim.close()
    o.lib.orc_build_cages(o.st)
    n = 24 ** 3
    rng = np.random.default_rng(3)
    xt = rng.standard_normal(n)
    xt -= xt.mean()
    b = np.zeros(n)
    dp = C.POINTER(C.c_double)
    o.lib.orc_poisson_apply(o.st, xt.ctypes.data_as(dp), b.ctypes.data_as(dp))
    assert abs(b.sum()) < 1e-9 * np.abs(b).sum()     # periodic: zero mean
    x = np.zeros(n)
    res = C.c_double()
    it = o.lib.orc_poisson_solve(o.st, b.ctypes.data_as(dp), x.ctypes.data_as(dp),
                                 1e-12, 5000, C.byref(res))
    assert it > 0 and res.value <= 1e-12
    x -= x.mean()
    assert np.abs(x - xt).max() < 1e-8 * np.abs(xt).max() * 1e3
    o.close()


# ---------------------------------------------------------------- BCs
def _walls_sim(tmp_path, n=(12, 10, 8)):
    d = str(tmp_path)
    configs.write_flow_config(os.path.join(d, "flow.config"), n=n,
                              lo=(0.0, 0.0, 0.0), hi=(1.2, 1.0, 0.8),
                              periodic=(True, True, False), nu=0.1)
    configs.write_part_config(os.path.join(d, "part.config"), [])
    return Sim(input_dir=d)


def test_boundary_ghosts_periodic_and_dirichlet(tmp_path):
    """x, y periodic (Gfx duplicates face is <-> ie-1), z no-slip walls:
    tangential ghost 8/3 bc - 2 u_ks + 1/3 u_ks+1, normal wall face = bc and
    ghost 2 bc - w_ks+1, Neumann pressure ghost = first interior plane
    (src/bluebottle_kernel.cu:145-154, 438-450, 1143-1156)."""
    sim = _walls_sim(tmp_path)
    d = sim.dom
    rng = np.random.default_rng(5)
    for nm in ("p", "u", "v", "w"):
        sim.array(nm)[:] = rng.standard_normal(sim.array(nm).size)
    o = Oracle.from_sim(sim, prepare=False)
    sim.close()
    o.lib.orc_dom_BC(o.st, 0)

    def arr(nm, G):
        return o.field(nm).reshape(G.knb, G.jnb, G.inb)

    u = arr("u", d.Gfx)
    w = arr("w", d.Gfz)
    p = arr("p", d.Gcc)
    ks = d.Gfx.ks
    # periodic in x for u: the ghost left of face `is` copies face ie-2, the
    # ghost right of ie-1 copies face is+1; faces is and ie-1 coincide
    G = d.Gfx
    isb, is_, ie, ieb = G.isb, getattr(G, "is"), G.ie, G.ieb
    inner = u[G.ks:G.ke, G.js:G.je]
    assert np.array_equal(inner[:, :, isb], inner[:, :, ie - 2])
    assert np.array_equal(inner[:, :, ieb - 1], inner[:, :, is_ + 1])
    # no-slip walls (bc value 0)
    assert np.allclose(u[G.ksb], -2.0 * u[ks] + u[ks + 1] / 3.0, rtol=0, atol=1e-14)
    Gz = d.Gfz
    assert np.all(w[Gz.ks] == 0.0)
    assert np.allclose(w[Gz.ksb], -w[Gz.ks + 1], rtol=0, atol=1e-14)
    assert np.all(w[Gz.ke - 1] == 0.0)
    assert np.allclose(p[d.Gcc.ksb], p[d.Gcc.ks], rtol=0, atol=0)
    o.close()


def test_projection_formula():
    """u = u* - dt/rho |flag_u| (phi_i - phi_i-1)/dx on every interior face
    (src/bluebottle_kernel.cu:1250-1302), no particles: |flag| = 1."""
    sim = Sim(configs.taylor_green(16))
    d = sim.dom
    rng = np.random.default_rng(11)
    us = rng.standard_normal(sim.array("u_star").size)
    ph = rng.standard_normal(sim.array("phi").size)
    sim.array("u_star")[:] = us
    sim.array("phi")[:] = ph
    o = Oracle.from_sim(sim, prepare=False)
    sim.close()
    o.lib.orc_build_cages(o.st)
    dt, rho = o.P.dt, o.P.rho_f
    o.lib.orc_project(o.st)
    u = o.field("u").reshape(d.Gfx.knb, d.Gfx.jnb, d.Gfx.inb)
    us3 = us.reshape(u.shape)
    ph3 = ph.reshape(d.Gcc.knb, d.Gcc.jnb, d.Gcc.inb)
    G = d.Gfx
    for k in range(G.ks, G.ke):
        for j in range(G.js, G.je):
            i = np.arange(getattr(G, "is"), G.ie)
            exp = us3[k, j, i] - dt / rho * (ph3[k, j, i] - ph3[k, j, i - 1]) / d.dx
            assert np.allclose(u[k, j, i], exp, rtol=0, atol=1e-13)
    o.close()
