"""GPU known-answer and wall-bounded parity cases, through the C ABI.

- The Stokes sphere of the reference's cuda_lamb_test
  (src/cuda_testing.cu:1836-2230): cuda_Lamb and cuda_part_BC on the
  analytic field reproduce the Stokes drag and the analytic face velocities,
  and agree with the oracle to round-off.
- A wall-bounded channel (x, y periodic, no-slip walls in z, driven by
  gradP.x) with two spheres: every field after three steps against the
  oracle, exercising the Dirichlet/Neumann boundary kernels and the
  non-periodic operator rows.
"""
import math
import os

import numpy as np
import pytest

from bluebottle_b200 import Sim, configs
from oracle.orc import Oracle
from tests.helpers import rel_err, field_interior, stokes_case, stokes_fields

pytestmark = pytest.mark.gpu


def test_stokes_sphere_on_gpu(gpu, tmp_path):
    W, a = 0.01, 1.0
    sim = stokes_case(tmp_path, n=48, L=3.0)
    fields = stokes_fields(sim, W=W, a=a)
    for nm, arr in fields.items():
        sim.array(nm)[:] = arr
    orc = Oracle.from_sim(sim, prepare=False)
    orc.lib.orc_build_cages(orc.st)
    orc.lib.orc_Lamb(orc.st)
    orc.lib.orc_part_BC(orc.st, 0)
    try:
        sim.prepare()
        for nm, arr in fields.items():        # undo the set-up's BC passes
            sim.array(nm)[:] = arr
        lib = sim.lib
        lib.cuda_dom_push()
        lib.cuda_Lamb()
        lib.cuda_part_BC()
        sim.pull()
        g, c = sim.parts()[0], orc.field("parts")[0]
        drag = 6.0 * math.pi * 1.0 * a * W
        assert abs(g.Fz - drag) / drag < 2e-3
        assert abs(g.Fz - c.Fz) <= 1e-12 * drag
        for k in ("Fx", "Fy", "Lx", "Ly", "Lz"):
            assert abs(getattr(g, k) - getattr(c, k)) < 1e-14, k
        # the modes the Stokes field does not excite are round-off (~1e-19):
        # compare every coefficient on the scale of the largest one
        names = ("pnm_re", "phinm_re", "chinm_re", "pnm_im", "phinm_im", "chinm_im")
        scale = max(np.abs(orc.field(nm)).max() for nm in names)
        for nm in names:
            e = np.abs(sim.array(nm) - orc.field(nm)).max()
            assert e <= 1e-12 * scale, nm
        for nm in ("u", "v", "w"):
            got = sim.array(nm)
            assert np.array_equal(sim.array("flag_" + nm), orc.field("flag_" + nm))
            assert np.abs(got - orc.field(nm)).max() < 1e-14
            set_ = got != fields[nm]
            assert set_.sum() > 100
            assert np.abs(got - fields[nm])[set_].max() < 3e-5
    finally:
        sim.close()
        orc.close()


def _channel(tmp_path, implicit=1):
    d = str(tmp_path)
    configs.write_flow_config(os.path.join(d, "flow.config"), n=(32, 32, 32),
                              lo=(0.0, 0.0, 0.0), hi=(8.0, 8.0, 8.0),
                              periodic=(True, True, False), nu=0.1,
                              pp_residual=1e-10, lamb_max_iter=2,
                              gradP=(-0.5, 0.0, 0.0), g=(0.0, 0.0, -1.0))
    configs.write_part_config(os.path.join(d, "part.config"),
                              [dict(r=1.0, x=3.1, y=4.2, z=4.0, rho=2.0),
                               dict(r=1.0, x=6.0, y=2.5, z=3.2, rho=1.5)])
    return Sim(input_dir=d, options=dict(fixed_dt=0.05, implicit=implicit,
                                         lamb_max_iter_override=2))


@pytest.mark.parametrize("implicit", [1, 0])
def test_wall_channel_with_spheres_parity(gpu, tmp_path, implicit):
    sim = _channel(tmp_path, implicit)
    orc = Oracle.from_sim(sim)
    try:
        sim.prepare()
        for _ in range(3):
            sim.step()
            orc.step()
        sim.pull()
        d = sim.dom
        for nm in ("phase", "phase_shell", "flag_u", "flag_v", "flag_w"):
            assert np.array_equal(sim.array(nm), orc.field(nm)), nm
        for nm in ("u", "v", "w", "p"):
            e = rel_err(field_interior(d, nm, sim.array(nm)),
                        field_interior(d, nm, orc.field(nm)))
            assert e < 1e-7, (nm, e)
        gp, cp = sim.parts(), orc.field("parts")
        for q in range(2):
            for k in ("x", "y", "z", "u", "v", "w", "Fx", "Fz"):
                a, b = getattr(gp[q], k), getattr(cp[q], k)
                assert abs(a - b) <= 1e-7 * max(1.0, abs(b)), (q, k, a, b)
        # the walls hold: no flow through z = 0 and z = 8
        w = sim.array("w").reshape(d.Gfz.knb, d.Gfz.jnb, d.Gfz.inb)
        assert np.all(w[d.Gfz.ks] == 0.0) and np.all(w[d.Gfz.ke - 1] == 0.0)
    finally:
        sim.close()
        orc.close()
