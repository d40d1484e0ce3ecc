"""Child process of test_gpu_refkernels.py's timing test: the reference's own
CUDA kernels (oracle/_ref/libref_gpu.so, the explicit build) and this
library side by side on one B200, each entry point of the time step that
the reference can run without CUSP called on the same state by both, and
timed on the host around a device-wide synchronisation (the reference's
entry points run on the legacy default stream and synchronise inside).

usage: python refgpu_time_child.py RUNDIR OUT.json
"""
import ctypes as C
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from bluebottle_b200 import abi  # noqa: E402
from tests.refgpu_child import Side, copy_state  # noqa: E402

ENTRY = ["cuda_build_cages", "cuda_dom_BC", "cuda_U_star_2", "cuda_part_BC_star",
         "cuda_dom_BC_star", "cuda_solvability", "cuda_dom_BC_phi", "cuda_project",
         "cuda_part_BC", "cuda_update_p", "cuda_part_p_fill", "cuda_dom_BC_p",
         "cuda_move_parts_sub", "cuda_Lamb", "cuda_lamb_err", "cuda_move_parts",
         "cuda_parts_internal", "cuda_store_u", "cuda_store_coeffs", "cuda_find_dt"]
RET = ("cuda_lamb_err", "cuda_find_dt")
REPS = 5


def main():
    run, out = sys.argv[1], sys.argv[2]
    lib = abi.load()
    reflib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so"),
                    mode=os.RTLD_LOCAL | getattr(os, "RTLD_DEEPBIND", 0))
    cudart = None
    for path in ("/usr/local/cuda/lib64/libcudart.so.12", "libcudart.so.12"):
        try:
            cudart = C.CDLL(path)
            break
        except OSError:
            continue
    os.chdir(run)
    lib.bbb_set_exit_on_failure(0)
    opts = abi.Options()
    lib.bbb_default_options(C.byref(opts))
    opts.implicit = 0
    lib.bbb_set_options(C.byref(opts))
    ref, ours = Side(reflib), Side(lib)
    reflib.domain_read_input()
    reflib.parts_read_input(0)
    for f in ("domain_init", "parts_init", "binDom_init"):
        getattr(reflib, f).restype = C.c_int
        assert getattr(reflib, f)() == 0, f
    assert lib.bbb_read_input(b"input") == 0
    assert lib.bbb_domain_init() == 0
    assert lib.bbb_parts_init() == 0
    rng = np.random.default_rng(5)
    for k, a in ref.arrays().items():
        if a.dtype.kind == "f":
            a[:] = 0.05 * rng.standard_normal(a.size)
        else:
            a[:] = -1 if k == "phase" else 1
    for k, v in (("dt", 0.01), ("dt0", 0.01), ("ttime", 0.5)):
        ref.scalar(k).value = v
    copy_state(ref, ours)
    for s in (ref, ours):
        s.call("cuda_dom_malloc")
        s.call("cuda_part_malloc")
        s.push()
        s.call("cuda_build_cages")
    res = {"cells": int(ours.dom.Gcc.s3), "particles": ours.nparts(), "reps": REPS}
    for e in ENTRY:
        row = {}
        for name, s in (("reference", ref), ("library", ours)):
            rt = C.c_double if e in RET else None
            s.call(e, restype=rt)                       # warm
            cudart.cudaDeviceSynchronize()
            t0 = time.perf_counter()
            for _ in range(REPS):
                s.call(e, restype=rt)
            cudart.cudaDeviceSynchronize()
            row[name + "_ms"] = (time.perf_counter() - t0) * 1e3 / REPS
        res[e] = row
        assert lib.bbb_last_status() == 0, (e, lib.bbb_last_status())
    for s in (ref, ours):
        s.call("cuda_part_free")
        s.call("cuda_dom_free")
    with open(out, "w") as fh:
        json.dump(res, fh)


if __name__ == "__main__":
    main()
