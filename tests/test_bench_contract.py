"""bench.py's reference arm (whole FP64 CPU steps of the path's algorithm,
set up by the reference's own input readers, timed on the host cores)
prints one JSON line with the keys of the benchmark contract; it needs no
GPU.  The small workload keeps it to seconds."""
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_contract_line():
    t0 = time.perf_counter()
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl",
                        "reference", "--steps", "2", "--warmup", "0",
                        "--workload", "tiny"],
                       capture_output=True, text=True, timeout=900, cwd=ROOT)
    wall = time.perf_counter() - t0
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup",
              "ms_per_step", "higher_is_better", "dtype", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 == d["e2e"]["d2h_bytes_per_step"]
    assert d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["cpu_baseline"]["cores"] >= 1
    # the steps it reports were timed: their total fits in the arm's own
    # wall time, and value is steps over that total
    assert d["steps"] >= 1
    assert d["steps"] * d["ms_per_step"] / 1000.0 <= wall
    assert abs(d["value"] - 1000.0 / d["ms_per_step"]) <= 1e-9 * d["value"]
    assert d["config"]["bicgstab_iters_per_step"] > 0
