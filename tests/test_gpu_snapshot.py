"""Asynchronous output snapshot (bbb_snapshot_start / _finish): the host
arrays the reference's writers read (u, v, w, p, phase, parts) receive the
state at the start call even though steps ran on the device since, equal
byte for byte to what the blocking pulls deliver at that point."""
import numpy as np
import pytest

from bluebottle_b200 import Sim, configs

pytestmark = pytest.mark.gpu

ERR_STATE = 5
NAMES = ("u", "v", "w", "p", "phase")


def _host(sim):
    f = {nm: sim.array(nm).copy() for nm in NAMES}
    parts = bytes(memoryview(sim.parts()).cast("B")) if sim.nparts else b""
    return f, parts


def test_snapshot_holds_the_state_of_its_start(gpu):
    wl = configs.sedimentation((32, 32, 64), (8.0, 8.0, 16.0), 6, nu=0.1,
                               lamb_max_iter=2, seed=3)
    sim = Sim(wl)
    try:
        sim.prepare()
        lib = sim.lib
        assert lib.bbb_snapshot_finish() == ERR_STATE      # nothing started
        sim.step()
        sim.pull()                          # blocking pulls: the reference's way
        want_f, want_p = _host(sim)
        assert lib.bbb_snapshot_start() == 0
        assert lib.bbb_snapshot_busy() == 1
        assert lib.bbb_snapshot_start() == ERR_STATE       # one at a time
        sim.lib.bbb_clear_status()
        for _ in range(2):                  # the device moves on meanwhile
            sim.step()
        # scribble over the host arrays: finish must rewrite them
        for nm in NAMES:
            sim.array(nm)[:] = 0
        assert lib.bbb_snapshot_finish() == 0
        assert lib.bbb_snapshot_busy() == 0
        got_f, got_p = _host(sim)
        for nm in NAMES:
            assert np.array_equal(got_f[nm], want_f[nm]), nm
        assert got_p == want_p
        # the state after the later steps is a different one
        sim.pull()
        later, _ = _host(sim)
        assert not np.array_equal(later["u"], want_f["u"])
        # a second snapshot reuses the buffers
        assert lib.bbb_snapshot_start() == 0
        assert lib.bbb_snapshot_finish() == 0
        again, _ = _host(sim)
        assert np.array_equal(again["u"], later["u"])
        assert sim.status() == 0
    finally:
        sim.close()
