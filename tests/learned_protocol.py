"""The learned-guess protocol of the 256^3 sedimentation configuration,
through the library's C ABI on one GPU.

  python -m tests.learned_protocol [--gen-steps 2000] [--infer-steps 1000]

Periodic 256^3 box of side 64 radii, 2000 seeded spheres (density ratio 2,
gravity along -z), FP32 inner solves in FP64 defect correction to 1e-8,
3 Lamb sub-iterations per step.

Phase 1 (tuple generation): `--gen-steps` plain steps; the first Poisson
solve of each step records crops of its (features, converged correction)
tuple, and every `--train-every` steps the net takes `--train-iters` Adam
steps (lr 1e-3, MSE) on the recorded crops, so it is trained on tuples from
the whole phase.  A final `--final-iters` Adam steps close the phase.

Phase 2 (inference): `--infer-steps` steps that alternate: even steps start
their first solve from the learned guess wherever its FP64 residual is below
the extrapolation's (no cost gate), odd steps from the extrapolation
(phi of the previous solve, as the reference).  Neighbouring steps have
nearly the same solve difficulty, so the two halves compare the iterations
of the first solve with and without the net; every guess step also reports
both initial residuals.

Spheres are given Young's modulus `--E` (1e4 by default instead of the
reference's 1e6): with the contact forces integrated explicitly at the
flow's CFL time step, as the reference does, E = 1e6 throws a touching pair
apart within one step (its contact time is far below dt).  The Poisson
problem the guess acts on does not depend on E.  Even so the 256^3 run
does not reach 3000 steps: at step 434 (seed 1) the advective CFL number
jumps from 0.4 to 125 and the step fails on its time-step bound -- a pair
closer than the quadrature shell (rs = 1.2 a), whose nodes then lie inside
the partner, the failure the seeding gap of 0.5 a avoids at the start
(the 128^3 configuration meets it at step 276).  The phases are therefore
run shortened, `--gen-steps 250 --infer-steps 120`, inside that window.

One JSON object per step, then a summary object.
"""
import argparse
import ctypes as C
import json
import statistics
import sys

from bluebottle_b200 import Sim, configs


def _mean(xs):
    return statistics.fmean(xs) if xs else None


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gen-steps", type=int, default=2000)
    ap.add_argument("--infer-steps", type=int, default=1000)
    ap.add_argument("--train-every", type=int, default=50)
    ap.add_argument("--train-iters", type=int, default=100)
    ap.add_argument("--final-iters", type=int, default=1000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--E", type=float, default=1e4)
    ap.add_argument("--prec", type=int, default=1)
    ap.add_argument("--n", type=int, default=256,
                    help="cells per side (256: the benchmark configuration; "
                    "smaller values scale the box and sphere count with it)")
    args = ap.parse_args(argv)

    if args.n == 256:
        wl = configs.config_c4(prec=args.prec)
    else:
        side = args.n / 4.0
        npart = max(1, int(round(2000 * (args.n / 256.0) ** 3)))
        wl = configs.sedimentation((args.n,) * 3, (side,) * 3, npart, nu=0.05,
                                   prec=args.prec, gap=configs.DENSE_GAP,
                                   loa=configs.DENSE_LOA)
    sim = Sim(wl, options=dict(learned_guess=1, lamb_max_iter_override=3))
    out = sys.stdout
    try:
        for p in sim.parts():
            p.E = args.E
        sim.prepare()
        lib = sim.lib
        lib.bbb_learn_train.restype = C.c_double
        lib.bbb_learn_train.argtypes = [C.c_int, C.c_double]
        lib.bbb_mark_elapsed.restype = C.c_double

        def one(phase, k, mode):
            lib.bbb_learn_enable(mode)
            lib.bbb_mark(0)
            sim.step()
            lib.bbb_mark(1)
            st = sim.stats()
            rec = dict(phase=phase, step=k, ms=lib.bbb_mark_elapsed(0, 1),
                       dt=st.step_dt, cfl=st.cfl_adv,
                       iters_first=st.pp_iters_first,
                       iters_total=st.pp_iters_total, solves=st.pp_solves,
                       guess_evaluated=st.guess_evaluated,
                       guess_used=st.guess_used)
            if st.guess_evaluated:
                rec.update(guess_r0=st.guess_r0, extrap_r0=st.extrap_r0,
                           r0_ratio=(st.guess_r0 / st.extrap_r0
                                     if st.extrap_r0 > 0 else None),
                           guess_cost_ms=st.guess_cost_ms)
            return rec

        losses = []
        for k in range(args.gen_steps):
            rec = one("generate", k, 1)
            if (k + 1) % args.train_every == 0:
                rec["train_loss"] = lib.bbb_learn_train(args.train_iters, args.lr)
                losses.append(rec["train_loss"])
            print(json.dumps(rec), file=out, flush=True)
        final_loss = lib.bbb_learn_train(args.final_iters, args.lr)
        print(json.dumps(dict(phase="train", adam_steps=args.final_iters,
                              crops=lib.bbb_learn_crops(),
                              last_batch_rel_mse=final_loss)), file=out, flush=True)
        guess, plain = [], []
        for k in range(args.infer_steps):
            use = k % 2 == 0
            rec = one("infer_guess" if use else "infer_plain",
                      args.gen_steps + k, 2 if use else 0)
            (guess if use else plain).append(rec)
            print(json.dumps(rec), file=out, flush=True)
        ratios = [r["r0_ratio"] for r in guess if r.get("r0_ratio")]
        summary = dict(
            phase="summary", n=args.n, E=args.E, gen_steps=args.gen_steps,
            infer_steps=args.infer_steps,
            online_train_losses_first_last=[losses[0], losses[-1]] if losses else None,
            final_train_rel_mse=final_loss,
            guess_steps=len(guess), plain_steps=len(plain),
            guess_used_fraction=_mean([r["guess_used"] for r in guess]),
            mean_r0_ratio=_mean(ratios),
            median_r0_ratio=statistics.median(ratios) if ratios else None,
            iters_first_guess=_mean([r["iters_first"] for r in guess]),
            iters_first_plain=_mean([r["iters_first"] for r in plain]),
            iters_step_guess=_mean([r["iters_total"] for r in guess]),
            iters_step_plain=_mean([r["iters_total"] for r in plain]),
            guess_cost_ms=_mean([r["guess_cost_ms"] for r in guess
                                 if "guess_cost_ms" in r]),
            ms_step_guess=_mean([r["ms"] for r in guess]),
            ms_step_plain=_mean([r["ms"] for r in plain]))
        print(json.dumps(summary), file=out, flush=True)
    finally:
        sim.close()


if __name__ == "__main__":
    main()
