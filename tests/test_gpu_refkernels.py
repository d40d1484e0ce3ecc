"""This library's non-solver cuda_* entry points against the reference's own
CUDA kernels: the reference's src/*.cu (all but src/cuda_bicgstab.cu, which
needs CUSP) compiled unmodified for sm_100a into oracle/_ref/libref_gpu.so
(oracle/ref.mk, target gpu; both the default explicit build and the
-DIMPLICIT Crank-Nicolson build, libref_gpu_implicit.so, the latter against
the library's Crank-Nicolson form) and run side by side with the library in a
child process (tests/refgpu_child.py) through the explicit time step of
src/bluebottle.c:603-708; its pressure solve and the three Crank-Nicolson
Helmholtz solves are checked against the systems the reference's own
kernels assemble (oracle/ref_pp_shim.cu restates the assembly half of
src/cuda_bicgstab.cu's solves, whose other half is CUSP).  Every stage starts from
bit-identical host state on both sides; the reference's flag arrays, which
its cuda_part_pull copies only in a -DDDEBUG build, are read from its device
pointers.  Each stage must change something on the reference side (so an
entry point that did nothing on both sides cannot pass).

Tolerances: integer masks and cage indices are equal; FP64 results agree to
a few ulps of the largest value (the library sums in other orders: fused
stencils, warp reductions).  The reference's compute_error races between
particles (its scratch rows overlap), so the Lamb error it returns is
compared loosely."""
import json
import os
import subprocess
import sys

import pytest

from bluebottle_b200 import configs

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
from tests.helpers import REF_SRC as REFSRC  # noqa: E402
REFGPU = {"explicit": os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so"),
          "implicit": os.path.join(ROOT, "oracle", "_ref", "libref_gpu_implicit.so")}

REL = 1e-12          # FP64 agreement, relative to the largest magnitude


def _ensure(build):
    if os.path.isdir(REFSRC):
        subprocess.run(["make", "-s", "-j8", "-f", os.path.join(ROOT, "oracle", "ref.mk"),
                        "REF=" + REFSRC, "gpu"], check=True, cwd=ROOT)
    if not os.path.exists(REFGPU[build]):
        pytest.skip("oracle/_ref/%s was not built (needs the reference tree)"
                    % os.path.basename(REFGPU[build]))


CASES = {
    # z walls, 3 spheres
    "walls_z": dict(flow=dict(n=(32, 16, 24), hi=(8.0, 4.0, 6.0), periodic=(True, True, False)),
                    parts=[dict(r=0.8, x=3.0, y=2.0, z=3.0), dict(r=0.7, x=6.0, y=2.2, z=2.5),
                           dict(r=0.6, x=1.2, y=0.9, z=4.4)]),
    # triply periodic, spheres across the west, south and top faces
    "periodic": dict(flow=dict(n=(24, 20, 18), hi=(6.0, 5.0, 4.5), periodic=(True, True, True)),
                     parts=[dict(r=0.7, x=0.3, y=2.5, z=2.0), dict(r=0.6, x=3.0, y=0.2, z=2.2),
                            dict(r=0.65, x=4.2, y=3.4, z=4.3), dict(r=0.5, x=2.0, y=4.0, z=0.9)]),
    # x and y walls, an odd cell count along x
    "walls_xy": dict(flow=dict(n=(21, 24, 16), hi=(5.25, 6.0, 4.0), periodic=(False, False, True)),
                     parts=[dict(r=0.7, x=1.0, y=1.1, z=2.0), dict(r=0.6, x=4.0, y=4.5, z=0.4),
                            dict(r=0.5, x=2.6, y=3.0, z=3.0)]),
}


def _case(tmp_path, name):
    c = CASES[name]
    d = tmp_path / "run"
    (d / "input").mkdir(parents=True)
    configs.write_flow_config(str(d / "input" / "flow.config"), lo=(0.0, 0.0, 0.0),
                              nu=0.1, pp_residual=1e-10, lamb_max_iter=2,
                              g=(0.0, 0.0, -1.0), **c["flow"])
    configs.write_part_config(str(d / "input" / "part.config"),
                              [dict(q, rho=2.0) for q in c["parts"]])
    return d


@pytest.mark.parametrize("build", ["explicit", "implicit"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_entry_points_match_reference_kernels(gpu, tmp_path, case, build):
    _ensure(build)
    run = _case(tmp_path, case)
    out = tmp_path / "diff.json"
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "refgpu_child.py"),
                        str(run), str(out), build], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    res = json.load(open(out))
    bad = []
    # the library's pressure solve satisfies the reference's own assembled
    # system (src/cuda_bicgstab.cu:723-815 via oracle/ref_pp_shim.cu) to
    # the solver's tolerance (pp_residual 1e-10 on ||b||)
    pp = res.pop("PP_system")
    print("PP_system", json.dumps(pp))
    if not (pp["rel_resid"] <= 3e-10 and pp["rel_resid_start"] > 1e-6):
        bad.append(("PP_system", pp))
    # the Crank-Nicolson Helmholtz solves against the reference's assembled
    # u*, v*, w* systems (src/cuda_bicgstab.cu:44-712), same tolerance
    for c in "uvw":
        h = res.pop("helmholtz_" + c)
        print("helmholtz_" + c, json.dumps(h))
        if not (h["rel_resid"] <= 3e-10 and h["solution_vs_rhs"] > 1e-8):
            bad.append(("helmholtz_" + c, h))
    for stage, arrays in res.items():
        # the stage ran: it changed something on the reference side
        moved = [e.get("moved", 0.0) for e in arrays.values()]
        if stage not in ("find_dt", "energy") and max(moved) == 0:
            bad.append((stage, "nothing changed"))
        for name, e in arrays.items():
            if e["kind"] == "int":
                ok = e["d"] == 0
            elif name == "return.cuda_lamb_err":
                ok = True
            else:
                ok = e["d"] <= REL * max(e["mag"], 1e-300)
            if not ok:
                bad.append((stage, name, e))
    print(json.dumps(res))
    assert not bad, bad


def test_reference_kernels_timing(gpu, tmp_path):
    """The same entry points timed on both sides (tests/refgpu_time_child.py)
    on a 128^3 periodic box with 500 seeded spheres: a measurement printed
    for the record, not a pass criterion beyond both sides having run."""
    _ensure("explicit")
    from bluebottle_b200 import Sim
    d = tmp_path / "run"
    (d / "input").mkdir(parents=True)
    configs.write_flow_config(str(d / "input" / "flow.config"), n=(128, 128, 128),
                              hi=(32.0, 32.0, 32.0), nu=0.05, pp_residual=1e-8,
                              lamb_max_iter=3, g=(0.0, 0.0, -1.0))
    sim = Sim(configs.sedimentation((128, 128, 128), (32.0, 32.0, 32.0), 500, seed=3))
    try:
        sim.write_part_config(str(d / "input" / "part.config"))
    finally:
        sim.close()
    out = tmp_path / "time.json"
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "refgpu_time_child.py"),
                        str(d), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    res = json.load(open(out))
    print("TIMING", json.dumps(res))
    for k, row in res.items():
        if isinstance(row, dict):
            assert row["reference_ms"] > 0 and row["library_ms"] > 0, k
