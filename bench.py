#!/usr/bin/env python
"""Headline benchmark: timesteps/s of the bluebottle step at 256x256x512
cells with 8000 seeded spheres (periodic box 64x64x128 radii, density
ratio 2, gravity along -z, nu = 0.05), Crank-Nicolson + Helmholtz CG,
pressure-Poisson Jacobi-BiCGSTAB to 1e-8 relative residual, Physalis
coupling.  The measured form is FP32 inner solves inside FP64 defect
correction; the plain FP64 form runs on the same inputs for comparison.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 is launched with torch.distributed.run, one process per GPU; the
path does not shard (one GPU per simulation), so every rank runs an
independent replica and `value` counts the time steps of all ranks.
`--impl reference` times the reference's CPU algorithm (the FP64 C
restatement in oracle/, OpenMP on the host cores) on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("timesteps/s at 256x256x512+8000 spheres, learned/FP32 vs plain "
          "FP64, same tol")
LAMB_ITERS = 3          # Lamb sub-iterations per step, fixed for the bench
LEARN_ITERS = 200       # Adam steps of the learned guess before timing


def dist_env():
    return (int(os.environ.get("RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Dist:
    """Barrier and max over ranks; gloo over TCP (plumbing only)."""

    def __init__(self, world):
        self.world = world
        self.pg = None
        if world > 1:
            import torch.distributed as td
            from datetime import timedelta
            td.init_process_group("gloo", timeout=timedelta(seconds=900))
            self.td = td

    def barrier(self):
        if self.world > 1:
            self.td.barrier()

    def max(self, x):
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.td.destroy_process_group()


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.gpu = gpu_index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [q.strip() for q in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def workload(name, prec):
    from bluebottle_b200 import configs
    if name == "small":
        # the same sedimentation set-up at 1/8 the cells and spheres, for
        # profiler captures (each FP32 vector 16.8 MB, 10 of them > L2)
        wl = configs.sedimentation((128, 128, 256), (32.0, 32.0, 64.0), 1000,
                                   nu=0.05, prec=prec, lamb_max_iter=LAMB_ITERS)
    else:
        wl = configs.config_c5(prec=prec, lamb_max_iter=LAMB_ITERS)
    return wl


def profiler_range(on):
    """cuProfilerStart / cuProfilerStop on the current context: with
    `ncu --profile-from-start off` only the bracketed launches are seen"""
    import ctypes as C
    cu = C.CDLL("libcuda.so.1")
    (cu.cuProfilerStart if on else cu.cuProfilerStop)()


def run_form(prec, steps, warmup, e2e_steps, profile=True, wl_name="c5",
             learned=False, prof_range=False):
    """One fresh simulation of the workload in precision form `prec`.  With
    `learned`, the warm-up steps record training crops of the first Poisson
    solve of each step, the net is trained on them (outside the timed
    region), and the timed steps start that solve from the gated learned
    guess.  The evaluation itself is cost-gated (bbb_learn_enable bit 4):
    the untimed step after training measures the guess's cost and its
    estimated saving, and while the saving stays below the cost the guess
    is evaluated only every 8 .. 256 steps."""
    from bluebottle_b200 import Sim
    import ctypes as C
    wl = workload(wl_name, prec)
    sim = Sim(wl, options=dict(lamb_max_iter_override=LAMB_ITERS,
                               learned_guess=1 if learned else 0))
    lib = sim.lib
    sim.prepare()
    for _ in range(warmup):
        sim.step()
    out = {}
    if learned:
        lib.bbb_learn_train.restype = C.c_double
        lib.bbb_learn_train.argtypes = [C.c_int, C.c_double]
        out["learn_crops"] = lib.bbb_learn_crops()
        out["learn_loss"] = lib.bbb_learn_train(LEARN_ITERS, 1e-3)
        lib.bbb_learn_enable(2 | 4)
        sim.step()                 # one untimed step with the guess in use
        st = sim.stats()
        out["probe"] = dict(evaluated=st.guess_evaluated, used=st.guess_used,
                            cost_ms=st.guess_cost_ms,
                            benefit_ms=st.guess_benefit_ms,
                            r0_ratio=(st.guess_r0 / st.extrap_r0
                                      if st.extrap_r0 > 0 else None))
    used, evaluated, ratios = 0, 0, []
    solves = 0
    lib.bbb_profile_reset()
    lib.bbb_profile_enable(1 if profile else 0)
    launches0 = lib.bbb_kernel_launches()
    iters = 0                      # bbb_step resets its stats every step
    if prof_range:
        profiler_range(True)
    lib.bbb_mark(0)
    for _ in range(steps):
        sim.step()
        st = sim.stats()
        iters += st.pp_iters_total
        solves += st.pp_solves
        used += st.guess_used
        evaluated += st.guess_evaluated
        if st.guess_evaluated and st.extrap_r0 > 0 and st.guess_r0 > 0:
            ratios.append(st.guess_r0 / st.extrap_r0)
    lib.bbb_mark(1)
    if prof_range:
        profiler_range(False)
    out["guess_used_steps"] = used
    out["guess_evaluated_steps"] = evaluated
    out["guess_r0_ratio"] = (sum(ratios) / len(ratios)) if ratios else None
    ms = lib.bbb_mark_elapsed(0, 1)
    lib.bbb_profile_enable(0)
    out["ms"] = ms
    out["launches"] = lib.bbb_kernel_launches() - launches0
    out["pp_iters_per_step"] = iters / max(steps, 1)
    out["pp_iters_per_solve"] = iters / max(solves, 1)
    st = sim.stats()
    out["lamb_iters"] = st.lamb_iters
    out["outer"] = st.pp_outer_last
    pm, pi, pb = C.c_double(), C.c_longlong(), C.c_double()
    lib.bbb_profile_get(C.byref(pm), C.byref(pi), C.byref(pb))
    out["prof_ms"], out["prof_iters"], out["prof_bytes"] = pm.value, pi.value, pb.value
    for k in (0, 1):
        lib.bbb_profile_get_pass(k, C.byref(pm), C.byref(pi), C.byref(pb))
        out["pass%d" % k] = (pm.value, pi.value, pb.value)
    # end-to-end through the public API: particle records in from pinned
    # host memory, the step, particle records and dt back to the host
    n = sim.nparts
    rec = n * C.sizeof(sim.parts()[0].__class__) if n else 0
    e2e_iters = 0
    lib.bbb_mark(2)
    for _ in range(e2e_steps):
        lib.bbb_part_state_push()
        sim.step()
        lib.bbb_part_state_pull()
        _ = sim.scalar("dt")
        e2e_iters += sim.stats().pp_iters_total
    lib.bbb_mark(3)
    out["e2e_ms"] = lib.bbb_mark_elapsed(2, 3)
    # the end-to-end steps follow the timed ones, later in the run: their
    # iteration count is reported beside their rate
    out["e2e_iters_per_step"] = e2e_iters / max(e2e_steps, 1)
    out["e2e_h2d"] = rec
    out["e2e_d2h"] = rec + 8
    out["cells"] = sim.dom.xn * sim.dom.yn * sim.dom.zn
    out["nparts"] = n
    out["status"] = sim.status()
    sim.close()
    return out


def cpu_reference(samples_iters=(2, 6), pp_iters_per_step=None, threads=None):
    """Bounded CPU sample of the reference algorithm on the same workload:
    the FP64 Jacobi-BiCGSTAB of the oracle (13-diagonal DIA operator, OpenMP)
    on the 256x256x512 pressure system with the 8000-sphere identity rows.
    The per-iteration time comes from two truncated solves; timesteps/s is
    that time scaled by the GPU FP64 run's BiCGSTAB iterations per step (the
    rest of the step is excluded, so the CPU figure is an upper bound)."""
    import ctypes as C
    import numpy as np
    from bluebottle_b200 import Sim, configs
    from oracle.orc import Oracle
    wl = configs.config_c5(prec=0, lamb_max_iter=LAMB_ITERS)
    sim = Sim(wl)
    orc = Oracle.from_sim(sim, prepare=False)
    sim.close()
    lib = orc.lib
    if threads:
        lib.orc_set_threads(threads)
    cores = lib.orc_set_threads(0)
    lib.orc_build_cages(orc.st)
    n = orc.dom.xn * orc.dom.yn * orc.dom.zn
    rng = np.random.default_rng(1)
    b = rng.standard_normal(n)
    b -= b.mean()
    dp = C.POINTER(C.c_double)
    times = []
    for m in samples_iters:
        x = np.zeros(n)
        res = C.c_double()
        t0 = time.perf_counter()
        lib.orc_poisson_solve(orc.st, b.ctypes.data_as(dp), x.ctypes.data_as(dp),
                              1e-30, m, C.byref(res))
        times.append(time.perf_counter() - t0)
    orc.close()
    t_iter = (times[1] - times[0]) / (samples_iters[1] - samples_iters[0])
    return {"t_iter": t_iter, "cores": cores, "t_solves": times,
            "pp_iters_per_step": pp_iters_per_step}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-learned", action="store_true",
                    help="time the FP32 form without the learned initial guess")
    ap.add_argument("--profile-range", action="store_true",
                    help="bracket the timed steps of the FP32 form with "
                    "cuProfilerStart/Stop (for ncu --profile-from-start off)")
    ap.add_argument("--workload", default="c5", choices=["c5", "small"],
                    help="c5: the headline 256x256x512 + 8000 spheres; small: "
                    "128x128x256 + 1000 spheres for profiler captures")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if world > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    dist = Dist(world)
    peak, peak_kind = measured_peak()

    if args.impl == "reference":
        if rank == 0:
            fp64_iters = 600.0
            cpu = cpu_reference(pp_iters_per_step=fp64_iters)
            # each step is a bounded sample: steps x warmup are not re-run;
            # the sample above is the whole measurement
            v = 1.0 / (cpu["t_iter"] * fp64_iters)
            line = {"impl": "reference", "metric": METRIC, "value": v,
                    "unit": "timesteps/s", "n_gpus": args.gpus,
                    "steps": args.steps, "warmup": args.warmup,
                    "ms_per_step": 1000.0 / v, "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic (seeded sphere pack)",
                    "config": {"workload": "256x256x512 periodic, 8000 spheres r=1, "
                               "nu=0.05, tol 1e-8, CPU FP64 Jacobi-BiCGSTAB"},
                    "cpu_baseline": {"value": v, "unit": "timesteps/s",
                                     "cores": cpu["cores"], "kind": "port",
                                     "sample": "FP64 oracle BiCGSTAB, 2- and 6-iteration "
                                     "solves on the 33.5M-cell system; per-iteration time "
                                     "x %d iterations/step" % int(fp64_iters)},
                    "e2e": {"value": v, "unit": "timesteps/s",
                            "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        dist.close()
        return

    steps, warmup = args.steps, args.warmup
    sampler = ClockSampler(local if world > 1 else 0)
    dist.barrier()
    sampler.start()
    mixed = run_form(1, steps, warmup, e2e_steps=steps, wl_name=args.workload,
                     prof_range=args.profile_range,
                     learned=not args.no_learned)
    clocks = sampler.stop()
    ms = dist.max(mixed["ms"])
    e2e_ms = dist.max(mixed["e2e_ms"])
    fp64 = None
    if not args.no_fp64:
        fp64 = run_form(0, steps, 1, e2e_steps=0, profile=False,
                        wl_name=args.workload)
        fp64["ms"] = dist.max(fp64["ms"])
    dist.barrier()
    if rank == 0:
        value = world * steps / (ms / 1000.0)
        e2e_value = world * steps / (e2e_ms / 1000.0)
        # dominant kernel: pass A of the FP32 BiCGSTAB iteration
        a_ms, a_n, a_bytes = mixed["pass0"]
        achieved = a_bytes / (a_ms / 1000.0) / 1e9 if a_ms > 0 else None
        passes = {}
        for k, nm in ((0, "k_bicg_async<float,0>"), (1, "k_bicg_async<float,1>")):
            pms, pn, pby = mixed["pass%d" % k]
            passes[nm] = {"launches": pn, "ms_per_launch": pms / pn if pn else None,
                          "GB_s": pby / (pms / 1000.0) / 1e9 if pms > 0 else None}
        it_gbs = (mixed["prof_bytes"] / (mixed["prof_ms"] / 1000.0) / 1e9
                  if mixed["prof_ms"] > 0 else None)
        traffic = None
        tfile = os.path.join(ROOT, "profiles", "bicgstab_traffic.json")
        if os.path.exists(tfile):
            try:
                with open(tfile) as fh:
                    tj = json.load(fh)
                traffic = tj.get("pass_a_fp32_bytes_per_launch_full_scale")
            except Exception:
                traffic = None
        line = {"metric": METRIC, "value": value, "unit": "timesteps/s",
                "n_gpus": world, "steps": steps, "warmup": warmup,
                "ms_per_step": ms / steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
                "data": "synthetic (seeded sphere pack, splitmix64 seed 1)",
                "config": {"workload": ("256x256x512 periodic box 64x64x128, 8000 "
                                        if args.workload == "c5" else
                                        "128x128x256 periodic box 32x32x64, 1000 ")
                           + "spheres r=1 (6.4%), rho_p/rho_f=2, g=-1 z, nu=0.05, "
                           "CN+Helmholtz CG, Jacobi-BiCGSTAB tol 1e-8, FP32 inner "
                           "in FP64 defect correction",
                           "lamb_iters_per_step": LAMB_ITERS,
                           "learned_guess": None if args.no_learned else {
                               "train_crops": mixed.get("learn_crops"),
                               "adam_steps": LEARN_ITERS,
                               "last_batch_rel_mse": mixed.get("learn_loss"),
                               "timed_steps_guess_evaluated":
                                   mixed.get("guess_evaluated_steps"),
                               "timed_steps_guess_used": mixed.get("guess_used_steps"),
                               "timed_guess_r0_over_extrapolation_r0":
                                   mixed.get("guess_r0_ratio"),
                               "probe_step": mixed.get("probe")},
                           "bicgstab_iters_per_step": mixed["pp_iters_per_step"],
                           "bicgstab_iters_per_solve": mixed["pp_iters_per_solve"],
                           "cell_updates_per_s": value * mixed["cells"],
                           "fp64_bicgstab_iters_per_step":
                               fp64["pp_iters_per_step"] if fp64 else None,
                           "l2": "inputs larger than L2 (each vector 134 MB FP32)",
                           "parallelism": "replicas" if world > 1 else "1 GPU"},
                "gpu_launches": mixed["launches"],
                "clocks": clocks,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                             "unit": "GB/s",
                             "frac": achieved / peak if achieved else None,
                             "traffic": traffic,
                             "kernel": "k_bicg_async<float,0> (BiCGSTAB pass A, "
                             "FP32, inputs staged by tensor-map copies): "
                             "algorithmic 10 words + 1 mask byte per unknown",
                             "peak_kind": peak_kind,
                             "passes": passes,
                             "iteration_GB_s": it_gbs},
                "e2e": {"value": e2e_value, "unit": "timesteps/s",
                        "h2d_bytes_per_step": mixed["e2e_h2d"],
                        "d2h_bytes_per_step": mixed["e2e_d2h"],
                        "bicgstab_iters_per_step": mixed["e2e_iters_per_step"]}}
        if fp64:
            fv = world * steps / (fp64["ms"] / 1000.0)
            line["fp64_value"] = fv
            line["speedup_vs_fp64"] = value / fv
        if world == 1 and not args.no_cpu:
            try:
                cpu = cpu_reference(pp_iters_per_step=(fp64 or mixed)["pp_iters_per_step"])
                cv = 1.0 / (cpu["t_iter"] * (fp64 or mixed)["pp_iters_per_step"])
                line["cpu_baseline"] = {
                    "value": cv, "unit": "timesteps/s", "cores": cpu["cores"],
                    "kind": "port",
                    "sample": "FP64 oracle Jacobi-BiCGSTAB (DIA, OpenMP), 2- and "
                    "6-iteration solves on the same 33.5M-cell system; "
                    "per-iteration time x the GPU FP64 run's %.0f iterations/step"
                    % (fp64 or mixed)["pp_iters_per_step"]}
            except Exception as e:  # reported, not fatal
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
