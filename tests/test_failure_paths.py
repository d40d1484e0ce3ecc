"""Failure paths, made on the host: truncated input files, a Krylov
iteration cap of one, a NaN written into the host fields before they are
pushed.  Each failing call must return its status code promptly (no
solve runs on to its cap, nothing exits the process) and leave the
library usable for the next set-up.  The reference prints and exits on a
solver failure (src/cuda_bicgstab.cu:293-296, 1029-1032); the library
records the status instead while exit-on-failure is off."""
import os
import time

import numpy as np
import pytest

from bluebottle_b200 import Sim, abi, configs
from bluebottle_b200.sim import BBBError

ERR_NOT_CONVERGED, ERR_CONFIG, ERR_NONFINITE = 2, 3, 8


@pytest.mark.parametrize("keep", [0.3, 0.6, 0.95])
def test_truncated_flow_config_is_a_config_error(tmp_path, keep):
    d = str(tmp_path)
    configs.write_flow_config(os.path.join(d, "flow.config"), n=(16, 16, 16),
                              hi=(4.0, 4.0, 4.0))
    configs.write_part_config(os.path.join(d, "part.config"), [])
    path = os.path.join(d, "flow.config")
    text = open(path).read()
    open(path, "w").write(text[:int(len(text) * keep)])
    with pytest.raises(BBBError, match="read_input"):
        Sim(input_dir=d)
    lib = abi.load()
    assert lib.bbb_last_status() == ERR_CONFIG
    lib.bbb_host_free()
    lib.bbb_clear_status()


def test_truncated_part_config_is_a_config_error(tmp_path):
    d = str(tmp_path)
    configs.write_flow_config(os.path.join(d, "flow.config"), n=(16, 16, 16),
                              hi=(4.0, 4.0, 4.0))
    configs.write_part_config(os.path.join(d, "part.config"),
                              [dict(r=0.5, x=1.0, y=1.0, z=1.0),
                               dict(r=0.5, x=3.0, y=3.0, z=3.0)])
    path = os.path.join(d, "part.config")
    text = open(path).read()
    open(path, "w").write(text[:int(len(text) * 0.7)])
    with pytest.raises(BBBError, match="read_input"):
        Sim(input_dir=d)
    lib = abi.load()
    assert lib.bbb_last_status() == ERR_CONFIG
    lib.bbb_host_free()
    lib.bbb_clear_status()


def _sim(prec):
    wl = configs.sedimentation((64, 32, 32), (16.0, 8.0, 8.0), 3, nu=0.1,
                               lamb_max_iter=1, seed=4, prec=prec)
    sim = Sim(wl, options=dict(lamb_max_iter_override=1))
    sim.prepare()
    return sim


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_iteration_cap_of_one_reports_not_converged(gpu, prec):
    """pp_max_iter = 1: the pressure solve stops after one iteration (one
    inner sweep in the mixed form, whose sweeps share the cap) and reports
    BBB_ERR_NOT_CONVERGED."""
    sim = _sim(prec)
    try:
        sim.step()                               # a normal step first
        assert sim.status() == 0
        sim.set_scalar("pp_max_iter", 1)
        t0 = time.perf_counter()
        sim.lib.cuda_PP_bicgstab(0)
        dt = time.perf_counter() - t0
        assert sim.status() == ERR_NOT_CONVERGED
        st = sim.stats()
        assert st.pp_iters_last <= 2, st.pp_iters_last
        assert st.pp_outer_last <= 2
        assert dt < 5.0
    finally:
        sim.close()
        sim.lib.bbb_clear_status()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_nan_in_u_star_reports_nonfinite(gpu, prec):
    """A NaN written into the host u* and pushed: the pressure solve's
    right-hand side norm is not finite, so the solve stops at its set-up
    with BBB_ERR_NONFINITE instead of iterating to the cap."""
    sim = _sim(prec)
    try:
        sim.pull()
        us = sim.array("u_star")
        G = sim.dom.Gfx
        us[getattr(G, "is") + 3 + 5 * G.s1b + 7 * G.s2b] = np.nan
        sim.lib.cuda_dom_push()
        t0 = time.perf_counter()
        sim.lib.cuda_PP_bicgstab(0)
        dt = time.perf_counter() - t0
        assert sim.status() == ERR_NONFINITE
        assert sim.stats().pp_iters_last <= 1
        assert dt < 5.0
    finally:
        sim.close()
        sim.lib.bbb_clear_status()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_nan_in_velocity_stops_the_step(gpu, prec):
    """A NaN in the host velocity (w and its previous-step copy w0, which the
    momentum right-hand side reads), pushed: the step's first Helmholtz
    solve meets it and the step returns BBB_ERR_NONFINITE within seconds; a
    fresh simulation afterwards runs normally."""
    sim = _sim(prec)
    try:
        sim.pull()
        G = sim.dom.Gfz
        c = getattr(G, "is") + 2 + 4 * G.s1b + 6 * G.s2b
        sim.array("w")[c] = np.nan
        sim.array("w0")[c] = np.nan
        sim.lib.cuda_dom_push()
        t0 = time.perf_counter()
        with pytest.raises(BBBError):
            sim.step()
        assert time.perf_counter() - t0 < 10.0
        assert sim.status() == ERR_NONFINITE
    finally:
        sim.close()
        sim.lib.bbb_clear_status()
    again = _sim(prec)
    try:
        again.step()
        assert again.status() == 0
    finally:
        again.close()
