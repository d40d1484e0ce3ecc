#!/usr/bin/env python
"""Headline benchmark: timesteps/s of the bluebottle step at 256x256x512
cells with 8000 seeded spheres (periodic box 64x64x128 radii, density
ratio 2, gravity along -z, nu = 0.05), Crank-Nicolson + Helmholtz CG,
pressure-Poisson Jacobi-BiCGSTAB to 1e-8 relative residual, Physalis
coupling.  The measured form is FP32 inner solves inside FP64 defect
correction with the learned initial guess; the plain FP64 form runs on the
same inputs, over the same step numbers, for comparison.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 is launched with torch.distributed.run, one process per GPU; the
path does not shard (one GPU per simulation), so every rank runs an
independent replica and `value` counts the time steps of all ranks.
`--impl reference` times whole CPU steps of the reference's algorithm (the
FP64 C restatement in oracle/, OpenMP on the host cores), set up by the
reference's own input readers and initialisation, on the same workload.
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
LEARN_ONLINE = 100      # Adam steps of the learned guess after each
                        # warm-up step (on the crops recorded so far)
LEARN_ITERS = 1000      # Adam steps after the warm-up, before timing
LEARN_CROPS = 32        # training crops (128 x 32 x 32) recorded per
                        # warm-up step, 12.5% of the 256x256x512 box
PROBE_STEPS = 1         # untimed steps after the warm-up (the learned
                        # guess's cost probe); both forms take them, so both
                        # time the same step numbers
REF_STEPS = 2           # whole CPU steps the reference arm times at most

# kernel kinds timed live (bbb_profile_get_pass numbering) and their names
# in the FP32-inner form
KERNELS = ((0, "k_bicg_async<float,0>", "BiCGSTAB pass A (FP32): reads r, t, "
            "p, v, x, rh, mask (s = r - alpha v formed in registers); writes "
            "r, x, p, v: 10 words + 1 mask byte"),
           (1, "k_bicg_async<float,1>", "BiCGSTAB pass B (FP32): reads r, v, "
            "rh, mask; writes t: 4 words + 1 mask byte"),
           (2, "k_bicg_async<double,2>", "FP64 outer residual: reads x, b "
            "(FP64), mask; writes r (FP32): 21 bytes"),
           (3, "k_bicg_async<float,3>", "Helmholtz CG stencil pass (FP32, "
            "staged like the BiCGSTAB passes): reads r, p, mask; writes p, Ap: "
            "4 words + 1 byte"),
           (4, "k_cg2<float>", "Helmholtz CG pointwise pass (FP32): reads p, "
            "x, Ap, r, mask; writes x, r: 6 words + 1 byte"),
           (5, "k_star_rhs_z<C>", "Crank-Nicolson momentum RHS (FP64), one "
            "component per launch: u0, v0, w0, p0, conv0 read, u*, conv "
            "written: 7 words"))

WORKLOADS = {
    "c5": "256x256x512 periodic box 64x64x128, 8000 spheres",
    "small": "128x128x256 periodic box 32x32x64, 1000 spheres",
    "tiny": "64x64x64 periodic box 16x16x16, 8 spheres",
}


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
                                   nu=0.05, prec=prec, lamb_max_iter=LAMB_ITERS,
                                   gap=configs.DENSE_GAP, loa=configs.DENSE_LOA)
    elif name == "tiny":
        wl = configs.sedimentation((64, 64, 64), (16.0, 16.0, 16.0), 8,
                                   nu=0.05, prec=prec, lamb_max_iter=LAMB_ITERS,
                                   gap=configs.DENSE_GAP, loa=configs.DENSE_LOA)
    else:
        wl = configs.config_c5(prec=prec, lamb_max_iter=LAMB_ITERS)
    return wl


def workload_text(name, form):
    return (WORKLOADS[name] + " r=1 seeded >= 0.5 r apart, rho_p/rho_f=2, "
            "g=-1 z, nu=%s, CN + Helmholtz CG, Jacobi-BiCGSTAB tol 1e-8, CFL 0.5 "
            "dt rule, lubrication l/a=1, %s" % ("0.05", form))


def profiler_range(on):
    """cuProfilerStart / cuProfilerStop on the current context: with
    `ncu --profile-from-start off` only the bracketed launches are seen"""
    import ctypes as C
    cu = C.CDLL("libcuda.so.1")
    (cu.cuProfilerStart if on else cu.cuProfilerStop)()


def run_form(prec, steps, warmup, e2e_steps, profile=True, wl_name="c5",
             learned=False, prof_range=False, keep=False, lamb_pp_tol=0.0,
             gate=True, barrier=None):
    """One fresh simulation of the workload in precision form `prec`:
    `warmup` untimed steps, PROBE_STEPS untimed steps, `steps` timed steps
    and `e2e_steps` end-to-end steps.  With `learned`, the warm-up steps
    record training crops of the first Poisson solve of each step, the net
    is trained on them after each warm-up step and once more after the
    last (all outside the timed region), and the probe and timed
    steps start that solve from the gated learned guess.  The evaluation
    itself is cost-gated (bbb_learn_enable bit 4): the probe step measures
    the guess's cost and its estimated saving, and while the saving stays
    below the cost the guess is evaluated only every 8 .. 256 steps.
    With `keep` the simulation is returned open in out["sim"].  Each timed
    region is bracketed by a drained solver stream and `barrier` (the
    ranks' barrier under torchrun) on both sides."""
    from bluebottle_b200 import Sim
    import ctypes as C
    wl = workload(wl_name, prec)
    sim = Sim(wl, options=dict(lamb_max_iter_override=LAMB_ITERS,
                               learned_guess=1 if learned else 0,
                               lamb_pp_tol=lamb_pp_tol))
    lib = sim.lib

    def drain_and_barrier():
        # event slot 5: record and wait, so the stream is idle here
        lib.bbb_mark(5)
        lib.bbb_mark_elapsed(5, 5)
        if barrier is not None:
            barrier()

    sim.prepare()
    if learned:
        lib.bbb_learn_train.restype = C.c_double
        lib.bbb_learn_train.argtypes = [C.c_int, C.c_double]
        if lib.bbb_learn_set_crops_per_step(LEARN_CROPS) != 0:
            raise RuntimeError("bbb_learn_set_crops_per_step(%d)" % LEARN_CROPS)
    for _ in range(warmup):
        sim.step()
        if learned:
            lib.bbb_learn_train(LEARN_ONLINE, 1e-3)
    out = {}
    if learned:
        out["learn_crops"] = lib.bbb_learn_crops()
        out["learn_loss"] = lib.bbb_learn_train(LEARN_ITERS, 1e-3)
        lib.bbb_learn_enable(2 | 4 if gate else 2)
    for q in range(PROBE_STEPS):
        sim.step()
        if learned and q == 0:
            st = sim.stats()
            out["probe"] = dict(evaluated=st.guess_evaluated, used=st.guess_used,
                                cost_ms=st.guess_cost_ms,
                                benefit_ms=st.guess_benefit_ms,
                                r0_ratio=(st.guess_r0 / st.extrap_r0
                                          if st.extrap_r0 > 0 else None))
    used, evaluated, ratios = 0, 0, []
    solves, iters, helm, dts, cfls = 0, 0, 0, [], []
    lib.bbb_profile_reset()
    lib.bbb_profile_enable(1 if profile else 0)
    launches0 = lib.bbb_kernel_launches()
    if prof_range:
        profiler_range(True)
    drain_and_barrier()
    lib.bbb_mark(0)
    for _ in range(steps):
        sim.step()
        st = sim.stats()          # bbb_step resets its stats every step
        iters += st.pp_iters_total
        solves += st.pp_solves
        helm += st.helm_iters_total
        used += st.guess_used
        evaluated += st.guess_evaluated
        dts.append(st.step_dt)
        cfls.append(st.cfl_adv)
        if st.guess_evaluated and st.extrap_r0 > 0 and st.guess_r0 > 0:
            ratios.append(st.guess_r0 / st.extrap_r0)
    lib.bbb_mark(1)
    drain_and_barrier()
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
    out["helm_iters_per_step"] = helm / max(steps, 1)
    out["dt_range"] = [min(dts), max(dts)] if dts else None
    out["cfl_max"] = max(cfls) if cfls else None
    st = sim.stats()
    out["lamb_iters"] = st.lamb_iters
    out["outer"] = st.pp_outer_last
    pm, pi, pb = C.c_double(), C.c_longlong(), C.c_double()
    lib.bbb_profile_get(C.byref(pm), C.byref(pi), C.byref(pb))
    out["prof_ms"], out["prof_iters"], out["prof_bytes"] = pm.value, pi.value, pb.value
    for k, _, _ in KERNELS:
        lib.bbb_profile_get_pass(k, C.byref(pm), C.byref(pi), C.byref(pb))
        out["pass%d" % k] = (pm.value, pi.value, pb.value)
    # end-to-end through the public API: particle records in from pinned
    # host memory, the step, particle records and dt back to the host
    n = sim.nparts
    rec = n * C.sizeof(sim.parts()[0].__class__) if n else 0
    e2e_iters = 0
    # the host copy of the particle records is brought up to date once,
    # untimed: every timed end-to-end step then pushes the records the
    # previous one pulled
    lib.bbb_part_state_pull()
    drain_and_barrier()
    lib.bbb_mark(2)
    for _ in range(e2e_steps):
        lib.bbb_part_state_push()
        sim.step()
        lib.bbb_part_state_pull()
        _ = sim.scalar("dt")
        e2e_iters += sim.stats().pp_iters_total
    lib.bbb_mark(3)
    drain_and_barrier()
    out["e2e_ms"] = lib.bbb_mark_elapsed(2, 3)
    # the end-to-end steps follow the timed ones, later in the run: their
    # iteration count is reported beside their rate
    out["e2e_iters_per_step"] = e2e_iters / max(e2e_steps, 1)
    out["e2e_h2d"] = rec
    out["e2e_d2h"] = rec + 8
    out["cells"] = sim.dom.xn * sim.dom.yn * sim.dom.zn
    out["nparts"] = n
    out["status"] = sim.status()
    if keep:
        out["sim"] = sim
    else:
        sim.close()
    return out


def cpu_sample(sim):
    """Bounded CPU sample of the same workload at the state the GPU run
    reached: the FP64 oracle (the reference's discretisation, 13-diagonal
    Jacobi-BiCGSTAB and Jacobi-CG, OpenMP) takes one whole time step with
    one Lamb sub-iteration from the pulled device state; the timed steps
    run LAMB_ITERS sub-iterations, so the step time is scaled by that
    count (the once-per-step particle update and dt are a small part)."""
    from oracle.orc import Oracle
    sim.pull()
    orc = Oracle.from_sim(sim, prepare=False)
    try:
        orc.P.lamb_max_iter = 1
        cores = orc.lib.orc_set_threads(0)
        t0 = time.perf_counter()
        rc = orc.step()
        t = time.perf_counter() - t0
        st = orc.stats()
    finally:
        orc.close()
    return {"t_sub": t, "rc": rc, "cores": cores, "iters": st["pp_iters_total"]}


def reference_arm(args):
    """Whole FP64 CPU steps of the reference's algorithm on the workload:
    inputs written by oracle/seed.py, read and initialised by the
    reference's own src/domain.c and src/particle.c (oracle/_ref, -DIMPLICIT
    build), copied into the oracle, which takes min(--steps, REF_STEPS)
    timed steps (a CPU step needs no warm-up; one C5 step is about a
    minute and a half on 16 cores)."""
    import ctypes as C
    from oracle.orc import Oracle, reference_host_lib, reference_setup
    from oracle.seed import write_workload_inputs
    wl = workload(args.workload, 0)
    with tempfile.TemporaryDirectory(prefix="bbb_ref_") as d:
        write_workload_inputs(wl, os.path.join(d, "input"))
        if reference_host_lib(True) is not None:
            ref = reference_setup(d, implicit=True)
            orc = Oracle.from_reference(ref, implicit=1, lamb_override=LAMB_ITERS)
            ref.domain_clean()
            ref.parts_clean()
            setup = "the reference's own domain_read_input, parts_read_input, " \
                    "domain_init, parts_init (oracle/_ref/libref_host_implicit.so)"
        else:
            raise RuntimeError("oracle/_ref/libref_host_implicit.so is not built "
                               "(build() makes it where the reference tree exists)")
    cores = orc.lib.orc_set_threads(0)
    nsteps = max(1, min(args.steps, REF_STEPS))
    times, iters = [], 0
    for _ in range(nsteps):
        t0 = time.perf_counter()
        rc = orc.step()
        times.append(time.perf_counter() - t0)
        iters += orc.stats()["pp_iters_total"]
        if rc != 0:
            raise RuntimeError("oracle step failed (%d)" % rc)
    orc.close()
    total = sum(times)
    v = nsteps / total
    sample = ("%d whole FP64 time steps (%d Lamb sub-iterations each, "
              "Crank-Nicolson + Helmholtz Jacobi-CG, Jacobi-BiCGSTAB on the "
              "13-diagonal operator, Physalis coupling, particle update) from "
              "the initial state, timed one by one: %s s; set up by %s"
              % (nsteps, LAMB_ITERS, ", ".join("%.1f" % t for t in times), setup))
    return {"impl": "reference", "metric": METRIC, "value": v,
            "unit": "timesteps/s", "n_gpus": args.gpus, "steps": nsteps,
            "warmup": 0, "steps_requested": args.steps,
            "warmup_requested": args.warmup,
            "ms_per_step": 1000.0 * total / nsteps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded sphere pack, splitmix64 seed 1)",
            "config": {"workload": workload_text(args.workload,
                                                 "FP64 CPU oracle (OpenMP)"),
                       "lamb_iters_per_step": LAMB_ITERS,
                       "bicgstab_iters_per_step": iters / nsteps,
                       "cores": cores},
            "cpu_baseline": {"value": v, "unit": "timesteps/s", "cores": cores,
                             "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "timesteps/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def kernel_table(form, peak, fp64=False):
    """Per-kernel live timing of one form; in the FP64 form the Krylov
    kernels are the double instantiations and the words are 8 bytes."""
    rows = {}
    for k, name, what in KERNELS:
        pms, pn, pby = form["pass%d" % k]
        if pn <= 0 or pms <= 0:
            continue
        if fp64 and k in (0, 1, 3, 4):
            name = name.replace("float", "double")
            what = what.replace("FP32", "FP64")
        gbs = pby / (pms / 1000.0) / 1e9
        rows[name] = {"launches": pn, "ms_per_launch": pms / pn,
                      "GB_per_launch": pby / pn / 1e9, "GB_s": gbs,
                      "frac": gbs / peak, "bytes": what}
    return rows


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
    ap.add_argument("--no-gate", action="store_true",
                    help="evaluate the learned guess in every step (no cost "
                    "gate)")
    ap.add_argument("--lamb-pp-tol", type=float, default=0.0,
                    help="relative tolerance of the pressure solves of the "
                    "Lamb sub-iterations before the last (0: every solve to "
                    "1e-8, as the reference); applied to both forms")
    ap.add_argument("--workload", default="c5", choices=sorted(WORKLOADS),
                    help="c5: the headline 256x256x512 + 8000 spheres; small: "
                    "128x128x256 + 1000 spheres for profiler captures; tiny: "
                    "64^3 + 8 spheres for CPU checks")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if world > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)

    if args.impl == "reference":
        # rank 0 alone times the CPU path; the other ranks exit at once
        if rank == 0:
            print(json.dumps(reference_arm(args)), flush=True)
        return

    dist = Dist(world)
    peak, peak_kind = measured_peak()
    steps, warmup = args.steps, args.warmup
    sampler = ClockSampler(local if world > 1 else 0)
    dist.barrier()
    sampler.start()
    want_cpu = world == 1 and not args.no_cpu
    mixed = run_form(1, steps, warmup, e2e_steps=steps, wl_name=args.workload,
                     prof_range=args.profile_range,
                     learned=not args.no_learned, keep=want_cpu,
                     lamb_pp_tol=args.lamb_pp_tol, gate=not args.no_gate,
                     barrier=dist.barrier)
    clocks = sampler.stop()
    ms = dist.max(mixed["ms"])
    e2e_ms = dist.max(mixed["e2e_ms"])
    cpu = None
    if want_cpu:
        sim = mixed.pop("sim")
        try:
            cpu = cpu_sample(sim)
        except Exception as e:  # reported, not fatal
            cpu = {"error": str(e)[:300]}
        finally:
            sim.close()
    fp64 = None
    if not args.no_fp64:
        fp64 = run_form(0, steps, warmup, e2e_steps=0, wl_name=args.workload,
                        lamb_pp_tol=args.lamb_pp_tol, barrier=dist.barrier)
        fp64["ms"] = dist.max(fp64["ms"])
    dist.barrier()
    if rank == 0:
        value = world * steps / (ms / 1000.0)
        e2e_value = world * steps / (e2e_ms / 1000.0)
        kmixed = kernel_table(mixed, peak)
        top = kmixed.get("k_bicg_async<float,0>")
        achieved = top["GB_s"] if top else None
        it_gbs = (mixed["prof_bytes"] / (mixed["prof_ms"] / 1000.0) / 1e9
                  if mixed["prof_ms"] > 0 else None)
        traffic, traffic_source = None, None
        tfile = os.path.join(ROOT, "profiles", "bicgstab_traffic.json")
        if os.path.exists(tfile) and args.workload == "c5":
            try:
                with open(tfile) as fh:
                    tj = json.load(fh)
                traffic = tj.get("pass_a_fp32_bytes_per_launch_full_scale")
                traffic_source = "ncu capture, not this run: " + tj.get("source", tfile)
            except Exception:
                traffic = None
        form = ("FP32 inner BiCGSTAB/CG in FP64 defect correction, learned "
                "initial guess (cost-gated)" if not args.no_learned else
                "FP32 inner BiCGSTAB/CG in FP64 defect correction")
        line = {"metric": METRIC, "value": value, "unit": "timesteps/s",
                "n_gpus": world, "steps": steps, "warmup": warmup,
                "ms_per_step": ms / steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
                "data": "synthetic (seeded sphere pack, splitmix64 seed 1)",
                "config": {"workload": workload_text(args.workload, form),
                           "timed_steps": "steps %d..%d of the run (after %d "
                           "warm-up and %d probe steps)" % (
                               warmup + PROBE_STEPS + 1,
                               warmup + PROBE_STEPS + steps, warmup, PROBE_STEPS),
                           "lamb_iters_per_step": LAMB_ITERS,
                           "lamb_pp_tol": args.lamb_pp_tol or None,
                           "dt_range": mixed["dt_range"],
                           "cfl_max": mixed["cfl_max"],
                           "learned_guess": None if args.no_learned else {
                               "train_crops": mixed.get("learn_crops"),
                               "crops_per_warmup_step": LEARN_CROPS,
                               "adam_steps": LEARN_ITERS + LEARN_ONLINE * warmup,
                               "last_batch_rel_mse": mixed.get("learn_loss"),
                               "cost_gate": not args.no_gate,
                               "timed_steps_guess_evaluated":
                                   mixed.get("guess_evaluated_steps"),
                               "timed_steps_guess_used": mixed.get("guess_used_steps"),
                               "timed_guess_r0_over_extrapolation_r0":
                                   mixed.get("guess_r0_ratio"),
                               "probe_step": mixed.get("probe")},
                           "bicgstab_iters_per_step": mixed["pp_iters_per_step"],
                           "bicgstab_iters_per_solve": mixed["pp_iters_per_solve"],
                           "helmholtz_cg_iters_per_step": mixed["helm_iters_per_step"],
                           "cell_updates_per_s": value * mixed["cells"],
                           "fp64_bicgstab_iters_per_step":
                               fp64["pp_iters_per_step"] if fp64 else None,
                           "l2": "inputs larger than L2 (each FP32 vector "
                                 "%.0f MB)" % (mixed["cells"] * 4 / 1e6),
                           "parallelism": "replicas" if world > 1 else "1 GPU"},
                "gpu_launches": mixed["launches"],
                "clocks": clocks,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                             "unit": "GB/s",
                             "frac": achieved / peak if achieved else None,
                             "traffic": traffic,
                             "traffic_source": traffic_source,
                             "kernel": "k_bicg_async<float,0> (BiCGSTAB pass A, "
                             "FP32, inputs staged by tensor-map copies): "
                             "algorithmic 10 words + 1 mask byte per unknown",
                             "peak_kind": peak_kind,
                             "passes": kmixed,
                             "iteration_GB_s": it_gbs},
                "e2e": {"value": e2e_value, "unit": "timesteps/s",
                        "h2d_bytes_per_step": mixed["e2e_h2d"],
                        "d2h_bytes_per_step": mixed["e2e_d2h"],
                        "bicgstab_iters_per_step": mixed["e2e_iters_per_step"]}}
        if fp64:
            fv = world * steps / (fp64["ms"] / 1000.0)
            line["fp64_value"] = fv
            line["speedup_vs_fp64"] = value / fv
            line["fp64_kernels"] = kernel_table(fp64, peak, fp64=True)
        if cpu is not None:
            if "t_sub" in cpu:
                cv = 1.0 / (cpu["t_sub"] * LAMB_ITERS)
                line["cpu_baseline"] = {
                    "value": cv, "unit": "timesteps/s", "cores": cpu["cores"],
                    "kind": "port",
                    "sample": "FP64 CPU oracle (the reference's discretisation, "
                    "13-diagonal Jacobi-BiCGSTAB, OpenMP): one whole time step "
                    "with 1 Lamb sub-iteration from the state the GPU run "
                    "reached, %.1f s, %d BiCGSTAB iterations; x%d for the %d "
                    "sub-iterations of a timed step"
                    % (cpu["t_sub"], cpu["iters"], LAMB_ITERS, LAMB_ITERS)}
            else:
                line["cpu_baseline"] = {"value": None, "error": cpu.get("error")}
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
