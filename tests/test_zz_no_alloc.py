"""The allocation-free pressure solve against the regular entry point.

bbb_PP_bicgstab_static serves callers that cannot allocate device memory
(their own allocator owns the GPU, or their loop cannot take cudaMalloc's
device synchronisation).  Given the same u*, phase, flags and initial phi
it must produce the phi that cuda_PP_bicgstab produces, call after call,
although its scratch is one shared static device array.  This file is
collected last so a failure here cannot hide the other tests."""
import ctypes as C

import numpy as np
import pytest

from bluebottle_b200 import Sim, configs
from tests.helpers import rel_err, field_interior

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-9


def test_static_poisson_matches_entry_point(gpu):
    import torch
    wl = configs.sedimentation((32, 32, 32), (8.0, 8.0, 8.0), 4, nu=0.1,
                               tol=1e-10, lamb_max_iter=2, seed=11)
    sim = Sim(wl)
    lib = sim.lib
    try:
        sim.prepare()
        sim.step()          # nonzero u*, phi and particle rows
        sim.pull()
        d = sim.dom
        host = {k: sim.array(k).copy() for k in
                ("u_star", "v_star", "w_star", "phi", "phase", "flag_u",
                 "flag_v", "flag_w")}
        dev = {k: torch.from_numpy(v).to("cuda") for k, v in host.items()}
        per = [int(sim.bc.pW == 0), int(sim.bc.pS == 0), int(sim.bc.pB == 0)]
        stream = torch.cuda.current_stream().cuda_stream
        torch.cuda.synchronize()
        for call in range(2):
            # regular entry point on the library's own state
            sim.array("phi")[:] = host["phi"]
            lib.cuda_dom_push()
            lib.cuda_PP_bicgstab(0)
            assert sim.status() == 0
            lib.cuda_dom_pull()
            phi_ref = sim.array("phi").copy()
            # allocation-free variant on caller-owned buffers
            dev["phi"].copy_(torch.from_numpy(host["phi"]))
            torch.cuda.synchronize()
            iters, resid = C.c_int(), C.c_double()
            rc = lib.bbb_PP_bicgstab_static(
                d.xn, d.yn, d.zn, d.dx, d.dy, d.dz, per[0], per[1], per[2],
                dev["u_star"].data_ptr(), dev["v_star"].data_ptr(),
                dev["w_star"].data_ptr(), dev["phase"].data_ptr(),
                dev["flag_u"].data_ptr(), dev["flag_v"].data_ptr(),
                dev["flag_w"].data_ptr(), sim.scalar("rho_f"),
                sim.scalar("dt"), sim.scalar("pp_residual"),
                sim.scalar("pp_max_iter"), dev["phi"].data_ptr(),
                C.byref(iters), C.byref(resid), stream)
            assert rc == 0, rc
            assert resid.value <= sim.scalar("pp_residual")
            phi_new = dev["phi"].cpu().numpy()
            e = rel_err(field_interior(d, "phi", phi_new),
                        field_interior(d, "phi", phi_ref))
            assert e < FIELD_TOL, (call, e)
            assert iters.value == sim.stats().pp_iters_last
        # requests beyond the stated limit are refused, not attempted
        rc = lib.bbb_PP_bicgstab_static(
            128, 128, 128, 1., 1., 1., 1, 1, 1, None, None, None, None, None,
            None, None, 1., 1., 1e-8, 10, None, None, None, None)
        assert rc == 7
    finally:
        sim.close()
