"""The drop-in link itself: the reference's own host files (src/domain.c,
src/particle.c, src/rng.c, src/vtk.c), compiled unmodified and linked
against libbbb200.so (oracle/ref.mk, oracle/_ref/libref_dropin.so), read the
input files into this library's globals, hand them to its cuda_* entry
points and write the reference's VTK output from its host arrays -- what
src/bluebottle.c's program does with the library in place of its CUDA
files.  Each run is a child process (tests/dropin_child.py) so the two
set-ups never share a process's globals."""
import os
import subprocess
import sys

import numpy as np
import pytest

from bluebottle_b200 import configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
from tests.helpers import REF_SRC as REFSRC  # noqa: E402
DROPIN = os.path.join(ROOT, "oracle", "_ref", "libref_dropin.so")


def _ensure():
    if os.path.isdir(REFSRC):
        subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "ref.mk"),
                        "REF=" + REFSRC], check=True, cwd=ROOT)
    if not os.path.exists(DROPIN):
        pytest.skip("the reference tree is not available to build oracle/_ref")


def _case(tmp_path):
    d = tmp_path / "run"
    (d / "input").mkdir(parents=True)
    configs.write_flow_config(str(d / "input" / "flow.config"), n=(32, 16, 24),
                              lo=(0.0, 0.0, 0.0), hi=(8.0, 4.0, 6.0), nu=0.1,
                              periodic=(True, True, False), pp_residual=1e-10,
                              lamb_max_iter=2, g=(0.0, 0.0, -1.0))
    configs.write_part_config(str(d / "input" / "part.config"),
                              [dict(r=0.8, x=3.0, y=2.0, z=3.0, rho=2.0),
                               dict(r=0.7, x=6.0, y=2.2, z=2.5, rho=2.0)])
    return d


def _child(run, mode, out):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "dropin_child.py"),
                        str(run), mode, str(out)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return dict(np.load(str(out)))


def test_reference_setup_and_vtk_through_the_library(tmp_path):
    _ensure()
    run = _case(tmp_path)
    a = _child(run, "ref", tmp_path / "ref.npz")
    b = _child(run, "ours", tmp_path / "ours.npz")
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    # the reference's writer prints the library's host pressure with %e
    assert a["vtk_p"].size == a["p_inner"].size
    assert np.allclose(a["vtk_p"], a["p_inner"], rtol=6e-6, atol=0)


@pytest.mark.gpu
def test_reference_setup_runs_on_the_gpu(gpu, tmp_path):
    _ensure()
    run = _case(tmp_path)
    a = _child(run, "refrun", tmp_path / "ref.npz")
    b = _child(run, "oursrun", tmp_path / "ours.npz")
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert np.allclose(a["vtk_p"], a["p_inner"], rtol=6e-6, atol=1e-300)
    assert np.abs(a["w"]).max() > 0
