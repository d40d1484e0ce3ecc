"""The benchmark configurations against the FP64 CPU oracle, through the C
ABI: C1 (Taylor-Green 32^3, all 100 steps, both precision forms), C2 (64^3
+ 8 spheres) and C3 (128^3 + 256 spheres, FP32 inner solves) over a prefix
of their step counts.  The full-length runs are tests/baseline_runs.py run
as a script; their tables are kept with the profiles.

Tolerances: both sides stop every Krylov solve at ||r|| <= tol ||b||
(1e-10 for C1, 1e-8 for C2 and C3) from the same iterate; the fields may
differ by what that rule leaves, and the bound the fields and the
particles are held to is 1e-6 relative.  Integer masks are bit for bit
at every checkpoint."""
import math

import pytest

from tests.baseline_runs import oracle_run

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-6


def _check_rows(rows, field_tol, part_tol=FIELD_TOL, phi_tol=None):
    assert rows
    for r in rows:
        for nm in ("u", "v", "w", "p", "phi"):
            tol = phi_tol if (nm == "phi" and phi_tol) else field_tol
            assert r[nm] < tol, (r["step"], nm, r[nm])
        assert r["int_equal"], r["step"]
        for nm in ("u_p", "omega", "F", "L"):
            if nm in r:
                assert r[nm] < part_tol, (r["step"], nm, r[nm])
        if "x" in r:
            assert r["x"] < part_tol, (r["step"], r["x"])
        # both sides project onto a divergence-free field to the same rule
        assert r["div_max"] <= 10 * r["div_max_ref"] + 1e-12


@pytest.mark.parametrize("prec", [0, 1])
def test_c1_taylor_green_100_steps(gpu, prec):
    """C1: the whole run.  Fields to 1e-8 of the oracle (tol 1e-10); kinetic
    energy equal to the oracle's to 1e-10; early decay at the rate of the
    mode's discrete Laplacian eigenvalue, exp(-2 nu lambda t), and faster
    than that later (vortex stretching adds dissipation: 3.4e-3 below it at
    t = 1 in the oracle).  The pressure correction phi of a nearly steady
    pressure is small: relative to its own size the FP32-inner form's phi
    differs by up to 6e-6 (measured) while the fields agree to 1e-8, and
    the energy, quadratic in the fields, to 2e-9 (FP64 form: 1e-10)."""
    rows = oracle_run("c1", prec, 100, 10)
    _check_rows(rows, 1e-8, phi_tol=1e-9 if prec == 0 else 2e-5)
    dx = 2 * math.pi / 32
    lam = 3.0 * (2.0 / dx * math.sin(dx / 2)) ** 2
    e_tol = 1e-10 if prec == 0 else 2e-9
    for r in rows:
        assert abs(r["energy"] - r["energy_ref"]) <= e_tol * r["energy_ref"], (
            r["step"], r["energy"], r["energy_ref"])
        ratio = r["energy"] / r["energy0"] / math.exp(-2 * 0.01 * lam * r["time"])
        if r["step"] <= 10:
            assert abs(ratio - 1) < 2e-5, (r["step"], ratio)
        assert 1 - 5e-3 < ratio <= 1 + 2e-5, (r["step"], ratio)
        assert r["div_max"] < 1e-10


def test_c2_prefix_fp64(gpu):
    """C2, the first 20 of its 200 steps (FP64)."""
    rows = oracle_run("c2", 0, 20, 5)
    _check_rows(rows, FIELD_TOL)


def test_c3_prefix_fp32_inner(gpu):
    """C3, the first 2 of its 500 steps (the oracle takes about 40 s a
    step at 128^3), FP32 inner solves inside FP64 defect correction against
    the FP64 oracle."""
    rows = oracle_run("c3", 1, 2, 1)
    # phi, the step's pressure correction, is the solve's own unknown: its
    # relative difference is what the 1e-8 stopping rule leaves times the
    # system's conditioning (0.3-1.1e-6 measured); the fields u, v, w, p
    # built from it stay within 1e-6
    _check_rows(rows, FIELD_TOL, phi_tol=5e-6)
