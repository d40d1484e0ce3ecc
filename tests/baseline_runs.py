"""Parity runs of the benchmark configurations (C1 Taylor-Green 32^3, C2
64^3 + 8 spheres, C3 128^3 + 256 spheres) against the FP64 CPU oracle.

Test infrastructure: the -m gpu tests (tests/test_gpu_baseline_configs.py)
run short prefixes through `oracle_run`; the full-length runs are this
file run as a script on a GPU machine, e.g.

  python -m tests.baseline_runs oracle --config c2 --steps 200 --every 20
  python -m tests.baseline_runs forms --config c3 --steps 500 --every 50

`oracle` steps the library (through its C ABI) and the oracle from the
same host state and compares them every `every` steps: the velocity
components, the pressure and the pressure correction (max |a - b| / max |b|
over the interior), the divergence of both, the integer masks (bit for
bit) and every particle's position (absolute, in radii), velocity, angular
velocity, hydrodynamic force and torque (max difference over the largest
magnitude).  `forms` compares the library's FP32-inner form with its plain
FP64 form over the same steps, for runs too long for the CPU oracle.
Both print one JSON object per checkpoint and a markdown table.
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from bluebottle_b200 import Sim, configs, interior  # noqa: E402

FIELDS = (("u", "Gfx"), ("v", "Gfy"), ("w", "Gfz"), ("p", "Gcc"), ("phi", "Gcc"))
INTS = (("phase", "Gcc"), ("phase_shell", "Gcc"), ("flag_u", "Gfx"),
        ("flag_v", "Gfy"), ("flag_w", "Gfz"))
PART_GROUPS = (("x", ("x", "y", "z")), ("u_p", ("u", "v", "w")),
               ("omega", ("ox", "oy", "oz")), ("F", ("Fx", "Fy", "Fz")),
               ("L", ("Lx", "Ly", "Lz")))


def config(name, prec):
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
    raise ValueError(name)


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = float(np.max(np.abs(b))) if b.size else 0.0
    num = float(np.max(np.abs(a - b))) if b.size else 0.0
    return num / den if den > 0 else num


def divergence(dom, u, v, w, phase):
    """max |div u| over the fluid cells (phase -1), from the interior face
    arrays (k, j, i); the cells inside spheres carry the rigid-body fill."""
    du = (u[:, :, 1:] - u[:, :, :-1]) / dom.dx
    dv = (v[:, 1:, :] - v[:, :-1, :]) / dom.dy
    dw = (w[1:, :, :] - w[:-1, :, :]) / dom.dz
    div = np.abs(du + dv + dw)[phase < 0]
    return float(np.max(div)) if div.size else 0.0


def snapshot(dom, arrays, parts, nparts):
    """Interior fields, integer masks and particle vectors of one state.
    Face grids keep both end faces, so the divergence uses all of them."""
    s = {}
    for nm, g in FIELDS + INTS:
        s[nm] = interior(arrays(nm), getattr(dom, g)).copy()
    s["divmax"] = divergence(dom, s["u"], s["v"], s["w"], s["phase"])
    for grp, keys in PART_GROUPS:
        s[grp] = (np.array([[getattr(p, k) for k in keys] for p in parts])
                  if nparts else np.zeros((0, 3)))
    return s


def compare(a, b, box):
    """Errors of state a against state b (the reference side)."""
    e = {}
    for nm, _ in FIELDS:
        e[nm] = rel(a[nm], b[nm])
    e["div_max"] = a["divmax"]
    e["div_max_ref"] = b["divmax"]
    e["int_equal"] = all(np.array_equal(a[nm], b[nm]) for nm, _ in INTS)
    if len(b["x"]):
        d = a["x"] - b["x"]
        d -= box * np.round(d / box)          # a sphere that wrapped on one side
        e["x"] = float(np.max(np.abs(d)))
        for grp, _ in PART_GROUPS[1:]:
            e[grp] = rel(a[grp], b[grp])
    return e


def oracle_run(name, prec, steps, every, log=None, max_seconds=None):
    """Library (precision form `prec`) against the FP64 oracle for `steps`
    steps; returns the list of checkpoint rows."""
    from oracle.orc import Oracle
    wl = config(name, prec)
    sim = Sim(wl)
    orc = Oracle.from_sim(sim)
    rows = []
    t0 = time.perf_counter()
    try:
        sim.prepare()
        d = sim.dom
        box = np.array([d.xl, d.yl, d.zl])
        e0 = sim.energy()
        for k in range(1, steps + 1):
            sim.step()
            rc = orc.step()
            if rc != 0:
                raise RuntimeError("oracle step %d failed (%d)" % (k, rc))
            if k % every == 0 or k == steps:
                sim.pull()
                a = snapshot(d, sim.array, sim.parts(), sim.nparts)
                b = snapshot(d, orc.field, orc.field("parts"), orc.nparts)
                row = dict(config=name, prec=prec, step=k, time=sim.scalar("ttime"),
                           energy=sim.energy(), energy_ref=orc.energy(), energy0=e0,
                           iters=sim.stats().pp_iters_total,
                           iters_ref=orc.stats()["pp_iters_total"])
                row.update(compare(a, b, box))
                rows.append(row)
                if log:
                    print(json.dumps(row), file=log, flush=True)
            if max_seconds and time.perf_counter() - t0 > max_seconds:
                break
    finally:
        sim.close()
        orc.close()
    return rows


def form_states(name, prec, steps, every):
    wl = config(name, prec)
    sim = Sim(wl)
    out = {}
    try:
        sim.prepare()
        d = sim.dom
        for k in range(1, steps + 1):
            sim.step()
            if k % every == 0 or k == steps:
                sim.pull()
                out[k] = (snapshot(d, sim.array, sim.parts(), sim.nparts),
                          sim.scalar("ttime"), sim.energy())
        box = np.array([d.xl, d.yl, d.zl])
    finally:
        sim.close()
    return out, box


def forms_run(name, steps, every, log=None):
    """The FP32-inner form against the plain FP64 form of the library."""
    ref, box = form_states(name, 0, steps, every)
    mix, _ = form_states(name, 1, steps, every)
    rows = []
    for k in sorted(ref):
        a, ta, ea = mix[k]
        b, tb, eb = ref[k]
        row = dict(config=name, prec=1, against="library FP64", step=k,
                   time=ta, time_ref=tb, energy=ea, energy_ref=eb)
        row.update(compare(a, b, box))
        rows.append(row)
        if log:
            print(json.dumps(row), file=log, flush=True)
    return rows


def table(rows):
    cols = ["step", "u", "v", "w", "p", "phi", "div_max", "int_equal", "x",
            "u_p", "omega", "F", "L"]
    out = ["| " + " | ".join(cols) + " |", "|" + "---:|" * len(cols)]
    for r in rows:
        cells = []
        for c in cols:
            v = r.get(c)
            if isinstance(v, bool):
                cells.append("yes" if v else "NO")
            elif isinstance(v, float):
                cells.append("%.1e" % v)
            elif v is None:
                cells.append("-")
            else:
                cells.append(str(v))
        out.append("| " + " | ".join(cells) + " |")
    return "\n".join(out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["oracle", "forms"])
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c3"])
    ap.add_argument("--prec", type=int, default=0)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--every", type=int, default=5)
    ap.add_argument("--max-seconds", type=float, default=None)
    args = ap.parse_args()
    if args.mode == "oracle":
        rows = oracle_run(args.config, args.prec, args.steps, args.every,
                          log=sys.stdout, max_seconds=args.max_seconds)
    else:
        rows = forms_run(args.config, args.steps, args.every, log=sys.stdout)
    print(table(rows))
    if args.config == "c1" and rows:
        r = rows[-1]
        dx = 2 * math.pi / 32
        lam = 3.0 * (2.0 / dx * math.sin(dx / 2)) ** 2
        print("energy E/E0 %.10f, exp(-2 nu lambda t) %.10f"
              % (r["energy"] / r["energy0"], math.exp(-2 * 0.01 * lam * r["time"])))


if __name__ == "__main__":
    main()
