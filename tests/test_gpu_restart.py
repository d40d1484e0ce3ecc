"""A run restarted from the reference's restart file continues as the
uninterrupted run does (src/bluebottle.c:454-470: in_restart after the
device set-up, then cuda_dom_push / cuda_part_push)."""
import numpy as np
import pytest

from bluebottle_b200 import Sim, configs

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "p", "phi", "u0", "conv0_u", "w_star")
PART = ("x", "y", "z", "u", "v", "w", "ox", "oy", "oz", "Fx", "Fy", "Fz")


def _case():
    return configs.sedimentation((32, 32, 32), (8.0, 8.0, 8.0), 4, nu=0.1,
                                 tol=1e-10, lamb_max_iter=3, seed=7)


def _snapshot(sim):
    sim.pull()
    f = {k: sim.array(k).copy() for k in FIELDS}
    p = [{k: getattr(q, k) for k in PART} for q in sim.parts()]
    return f, p


def test_restart_continues_the_run(gpu, tmp_path):
    path = str(tmp_path / "restart.config")
    sim = Sim(_case())
    try:
        sim.prepare()
        for _ in range(2):
            sim.step()
        sim.pull()
        sim.out_restart(path)
        for _ in range(2):
            sim.step()
        want_f, want_p = _snapshot(sim)
        t_want = sim.scalar("ttime")
    finally:
        sim.close()

    sim = Sim(_case())
    try:
        sim.prepare()
        sim.in_restart(path)
        sim.push()
        assert sim.scalar("stepnum") == 2
        for _ in range(2):
            sim.step()
        got_f, got_p = _snapshot(sim)
        assert sim.scalar("ttime") == t_want
        for k in FIELDS:
            assert np.array_equal(got_f[k], want_f[k]), (k, float(np.max(np.abs(got_f[k] - want_f[k]))))
        for a, b in zip(got_p, want_p):
            assert a == b
    finally:
        sim.close()
