"""Per-step log of a benchmark workload through the library's C ABI.

  python -m bluebottle_b200.runlog --workload c5 --steps 120 [--prec 1]

One JSON object per step: the step's dt and advective CFL number, Lamb
sub-iterations and coefficient error, BiCGSTAB and Helmholtz CG iterations,
the device time of the step (CUDA events), and from the particle records
pulled after the step the closest surface gap (in radii), the largest
particle speed and the mean settling velocity.  Stops at the first step
that returns an error status and prints it.
"""
import argparse
import json
import sys

import numpy as np

from . import Sim, configs


def workload(name, prec):
    if name == "c1":
        wl = configs.config_c1()
        wl.options["precision"] = prec
        return wl
    if name == "c2":
        wl = configs.config_c2()
        wl.options["precision"] = prec
        return wl
    if name == "c3":
        return configs.config_c3(prec=prec)
    if name == "c4":
        return configs.config_c4(prec=prec)
    if name == "c5":
        return configs.config_c5(prec=prec, lamb_max_iter=3)
    if name == "small":
        return configs.sedimentation((128, 128, 256), (32.0, 32.0, 64.0), 1000,
                                     nu=0.05, prec=prec, lamb_max_iter=3,
                                     gap=configs.DENSE_GAP, loa=configs.DENSE_LOA)
    raise ValueError(name)


def min_gap(X, L, r):
    """Smallest surface gap over all pairs (periodic images), in radii."""
    from scipy.spatial import cKDTree
    Xm = np.mod(X, L)
    d, _ = cKDTree(Xm, boxsize=L).query(Xm, k=2)
    return float(d[:, 1].min() / r - 2.0)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c5",
                    choices=["c1", "c2", "c3", "c4", "c5", "small"])
    ap.add_argument("--prec", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--lamb-iters", type=int, default=3,
                    help="Lamb sub-iterations per step; 0 keeps the "
                    "workload's lamb_max_iter / lamb_residual rule")
    args = ap.parse_args(argv)
    wl = workload(args.workload, args.prec)
    sim = Sim(wl, options=dict(lamb_max_iter_override=max(args.lamb_iters, 0)))
    lib = sim.lib
    try:
        sim.prepare()
        d = sim.dom
        L = np.array([d.xl, d.yl, d.zl])
        for k in range(1, args.steps + 1):
            lib.bbb_mark(0)
            rc = lib.bbb_step()
            lib.bbb_mark(1)
            st = sim.stats()
            rec = dict(step=k, rc=rc, ms=round(lib.bbb_mark_elapsed(0, 1), 2),
                       dt=st.step_dt, cfl=st.cfl_adv, lamb_iters=st.lamb_iters,
                       lamb_err=st.lamb_err, bicgstab_iters=st.pp_iters_total,
                       bicgstab_iters_max=st.pp_iters_max,
                       outer_sweeps=st.pp_outer_last, resid=st.pp_resid_last,
                       cg_iters=st.helm_iters_total)
            if sim.nparts:
                lib.cuda_part_pull()
                P = sim.parts()
                X = np.array([[p.x, p.y, p.z] for p in P])
                U = np.array([[p.u, p.v, p.w] for p in P])
                rec.update(min_gap=min_gap(X, L, P[0].r),
                           max_speed=float(np.linalg.norm(U, axis=1).max()),
                           mean_w=float(U[:, 2].mean()))
            print(json.dumps(rec), flush=True)
            if rc != 0:
                print("status: %s" % lib.bbb_status_string(rc).decode(),
                      flush=True)
                return 1
    finally:
        sim.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
