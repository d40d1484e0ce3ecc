"""How much a better start saves the pressure-Poisson solve, measured on
the FP64 CPU oracle (the reference's discretisation and scaled
Jacobi-BiCGSTAB, src/cuda_bicgstab.cu:715-1073).

  python -m tests.poisson_start_study [--n 32 32 64] [--spheres 16] [--steps 8]

A periodic sedimentation box (4 cells per radius, spheres seeded 0.5 radii
apart, density ratio 2, nu = 0.05, tolerance 1e-8) steps through the
reference's sequence (src/bluebottle.c:603-708) with 3 Lamb sub-iterations
per step.  Before every Poisson solve it reports the initial residual of
the reference's start x0 = phi_prev relative to ||b||, and after it the
iterations and how far the solution moved from x0.  With `--coarse F` the
first solve of the last step is also started from phi_prev plus a
Galerkin coarse-grid correction (aggregates of F^3 fluid cells, the coarse
system solved exactly): the solve's iterations from both starts.

One JSON object per solve, then a summary object.
"""
import argparse
import ctypes as C
import json

import numpy as np

from bluebottle_b200 import Sim, configs
from oracle.orc import Oracle


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, nargs=3, default=[32, 32, 64])
    ap.add_argument("--spheres", type=int, default=16)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--coarse", type=int, default=0)
    args = ap.parse_args(argv)
    nx, ny, nz = args.n
    wl = configs.sedimentation((nx, ny, nz), (nx / 4.0, ny / 4.0, nz / 4.0),
                               args.spheres, nu=0.05, lamb_max_iter=3,
                               gap=configs.DENSE_GAP, loa=configs.DENSE_LOA)
    sim = Sim(wl)
    orc = Oracle.from_sim(sim)
    lib, st = orc.lib, orc.st
    n = nx * ny * nz
    dp = C.POINTER(C.c_double)

    def interior(name):
        a = orc.field(name).reshape(nz + 2, ny + 2, nx + 2)
        return a[1:-1, 1:-1, 1:-1].reshape(-1).copy()

    def apply(x):
        x = np.ascontiguousarray(x)
        y = np.zeros(n)
        lib.orc_poisson_apply(st, x.ctypes.data_as(dp), y.ctypes.data_as(dp))
        return y

    def solve(b, x0):
        x = np.ascontiguousarray(x0.copy())
        res = C.c_double()
        it = lib.orc_poisson_solve(st, b.ctypes.data_as(dp), x.ctypes.data_as(dp),
                                   orc.P.pp_residual, 20000, C.byref(res))
        return it

    rows = []
    coarse = None
    try:
        for s in range(args.steps):
            P = orc.P
            P.ttime += P.dt
            P.stepnum += 1
            lib.orc_compute_forcing(st)
            lib.orc_compute_vel_BC(st)
            lib.orc_build_cages(st)
            for sub in range(3):
                for c in range(3):
                    lib.orc_star_helmholtz(st, c)
                lib.orc_part_BC(st, 1)
                lib.orc_dom_BC(st, 1)
                lib.orc_solvability(st)
                lib.orc_part_BC(st, 1)
                lib.orc_dom_BC(st, 1)
                lib.orc_PP_rhs(st)
                lib.orc_part_BC_p(st)
                b = orc.field("rhs_p")[:n].copy()
                x0 = interior("phi")
                bn = np.linalg.norm(b)
                r0 = np.linalg.norm(b - apply(x0)) / bn
                if args.coarse and s == args.steps - 1 and sub == 0:
                    coarse = _coarse_compare(args.coarse, (nx, ny, nz),
                                             interior("phase"), apply, solve, b, x0)
                lib.orc_PP_bicgstab(st)
                xs = interior("phi")
                row = dict(step=s, sub=sub, iters=orc.stats()["pp_iters"],
                           r0_over_b=r0,
                           moved=float(np.linalg.norm(xs - x0) / np.linalg.norm(xs)))
                rows.append(row)
                print(json.dumps(row), flush=True)
                lib.orc_dom_BC(st, 2)
                lib.orc_project(st)
                lib.orc_part_BC(st, 0)
                lib.orc_dom_BC(st, 0)
                lib.orc_update_p(st)
                lib.orc_part_BC(st, 0)
                lib.orc_part_p_fill(st)
                lib.orc_dom_BC(st, 3)
                lib.orc_move_parts_sub(st)
                lib.orc_Lamb(st)
                lib.orc_lamb_err(st)
            lib.orc_move_parts(st)
            lib.orc_parts_internal(st)
            lib.orc_dom_BC(st, 0)
            lib.orc_store_u(st)
            lib.orc_store_coeffs(st)
            P.dt0 = P.dt
            P.dt = lib.orc_find_dt(st)
    finally:
        orc.close()
        sim.close()
    later = [r for r in rows if r["step"] > 0]
    summ = dict(summary=True, n=[nx, ny, nz], spheres=args.spheres)
    for sub in range(3):
        rs = [r for r in later if r["sub"] == sub]
        if rs:
            summ["sub%d" % sub] = dict(
                r0_over_b=[min(r["r0_over_b"] for r in rs),
                           max(r["r0_over_b"] for r in rs)],
                iters_mean=float(np.mean([r["iters"] for r in rs])))
    if coarse:
        summ["coarse"] = coarse
    print(json.dumps(summ), flush=True)


def _coarse_compare(F, dims, phase, apply, solve, b, x0):
    """phi_prev plus the Galerkin coarse-grid correction of its residual
    (piecewise-constant aggregates of F^3 cells, fluid cells only, the
    coarse system solved to 1e-12); iterations from both starts"""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    nx, ny, nz = dims
    cx, cy, cz = nx // F, ny // F, nz // F
    nc = cx * cy * cz
    fl = (phase < 0).astype(np.float64)

    def restrict(v):
        return (v * fl).reshape(cz, F, cy, F, cx, F).sum(axis=(1, 3, 5)).reshape(-1)

    def prolong(vc):
        v = vc.reshape(cz, cy, cx)
        return fl * np.repeat(np.repeat(np.repeat(v, F, 0), F, 1), F, 2).reshape(-1)

    # A_c = R A P column by column in groups: aggregates 4 apart along every
    # axis have disjoint stencil footprints (needs dimensions divisible by 4)
    CP = 4
    rows, cols, vals = [], [], []
    for oz in range(CP):
        for oy in range(CP):
            for ox in range(CP):
                sel = np.zeros((cz, cy, cx))
                sel[oz::CP, oy::CP, ox::CP] = 1.0
                yg = restrict(apply(prolong(sel.reshape(-1)))).reshape(cz, cy, cx)
                for kk, jj, ii in zip(*np.nonzero(yg)):
                    for dz in (-1, 0, 1):
                        z2 = (kk + dz) % cz
                        if (z2 - oz) % CP:
                            continue
                        for dy in (-1, 0, 1):
                            y2 = (jj + dy) % cy
                            if (y2 - oy) % CP:
                                continue
                            for dx in (-1, 0, 1):
                                x2 = (ii + dx) % cx
                                if (x2 - ox) % CP:
                                    continue
                                rows.append((kk * cy + jj) * cx + ii)
                                cols.append((z2 * cy + y2) * cx + x2)
                                vals.append(yg[kk, jj, ii])
    Ac = sp.csr_matrix((vals, (rows, cols)), shape=(nc, nc))
    r0 = b - apply(x0)
    ec = spl.lsqr(Ac, restrict(r0), atol=1e-12, btol=1e-12, iter_lim=50000)[0]
    x1 = x0 + prolong(ec - ec.mean())
    bn = np.linalg.norm(b)
    return dict(aggregate=F, coarse_cells=nc,
                r0_over_b=[float(np.linalg.norm(r0) / bn),
                           float(np.linalg.norm(b - apply(x1)) / bn)],
                iters=[solve(b, x0), solve(b, x1)])


if __name__ == "__main__":
    main()
