"""Build libbbb200.so (C host code + sm_100a CUDA kernels) in-tree.

Run as ``python -m bluebottle_b200.build``; nvcc cross-compiles for
sm_100a without a GPU present.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbbb200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".c")):
            out.append(os.path.join(CSRC, name))
    return out


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC)
                        if f.endswith((".h", ".cuh"))]
    deps += [os.path.join(HERE, "..", "include", f)
             for f in os.listdir(os.path.join(HERE, "..", "include"))]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    nvcc = _nvcc()
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17",
           "-Xcompiler", "-fPIC,-O2,-fno-strict-aliasing",
           "-Xptxas", "-O3", "--expt-relaxed-constexpr",
           "-shared", "-o", tmp, *sources(), *extra]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=HERE)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=[a for a in sys.argv[1:] if a.startswith("-D")])
    print(LIB)
