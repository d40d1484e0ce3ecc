"""Child process of test_gpu_refkernels.py: the reference's own CUDA kernels
(src/*.cu compiled unmodified for sm_100a into oracle/_ref/libref_gpu.so,
behind the reference's cuda_* entry points) and this library, side by side
in one process, through the entry points of src/bluebottle.c's time step
that do not need CUSP (everything but the Helmholtz and Poisson solves).

Both set up from the same input files with their own readers; the fields
are then filled with the same seeded values.  Before every stage the
reference's host state (fields, integer masks, particle records, Lamb
coefficients) is copied into this library's host arrays and both sides push,
so each stage starts from bit-identical inputs; after the stage both pull
and the child records, per array, the largest difference and the largest
reference magnitude.

usage: python refgpu_child.py RUNDIR OUT.json [explicit|implicit]
  explicit -- oracle/_ref/libref_gpu.so (the default build) and the library
              with its explicit Adams-Bashforth step
  implicit -- oracle/_ref/libref_gpu_implicit.so (-DIMPLICIT, the
              Crank-Nicolson program: no cuda_U_star_2, no diffusion
              histories, the implicit dt rule) and the library in its
              Crank-Nicolson form
"""
import ctypes as C
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from bluebottle_b200 import abi  # noqa: E402

FACE = {}
for c, g in zip("uvw", ("Gfx", "Gfy", "Gfz")):
    for pat in ("%s", "%s0", "%s_star", "diff0_%s", "conv0_%s", "diff_%s", "conv_%s"):
        FACE[pat % c] = g
CELL = {"p": "Gcc", "p0": "Gcc", "phi": "Gcc"}
INTS = {"phase": "Gcc", "phase_shell": "Gcc", "flag_u": "Gfx", "flag_v": "Gfy",
        "flag_w": "Gfz"}
COEF = ("pnm_re pnm_im pnm_re0 pnm_im0 pnm_re00 pnm_im00 phinm_re phinm_im "
        "phinm_re0 phinm_im0 phinm_re00 phinm_im00 chinm_re chinm_im "
        "chinm_re0 chinm_im0 chinm_re00 chinm_im00").split()
SCAL = ("dt", "dt0", "ttime")
# particle record members compared (bin is left unset by the reference
# until its collision pass bins the particles)
PSKIP = ("bin",)


class Side:
    def __init__(self, lib):
        self.lib = lib
        self.dom = abi.DomStruct.in_dll(lib, "Dom")

    def call(self, name, *args, restype=None):
        f = getattr(self.lib, name)
        f.restype = restype
        return f(*args)

    def arr(self, name, grid, ctype=C.c_double):
        """the host array (empty where the program does not allocate it:
        the -DIMPLICIT build has no diffusion histories)"""
        n = getattr(self.dom, grid).s3b
        ptr = C.POINTER(ctype).in_dll(self.lib, name)
        if not ptr:
            return np.zeros(0, np.float64 if ctype is C.c_double else np.int32)
        return np.ctypeslib.as_array(ptr, shape=(n,))

    def nparts(self):
        return C.c_int.in_dll(self.lib, "nparts").value

    def coef(self, name):
        n = self.nparts() * C.c_int.in_dll(self.lib, "coeff_stride").value
        return np.ctypeslib.as_array(C.POINTER(C.c_double).in_dll(self.lib, name),
                                     shape=(n,))

    def parts(self):
        pp = C.POINTER(abi.PartStruct).in_dll(self.lib, "parts")
        return (abi.PartStruct * self.nparts()).from_address(C.addressof(pp.contents))

    def scalar(self, name):
        return C.c_double.in_dll(self.lib, name)

    def arrays(self):
        out = {k: self.arr(k, g) for k, g in FACE.items()}
        out.update({k: self.arr(k, g) for k, g in CELL.items()})
        out.update({k: self.arr(k, g, C.c_int) for k, g in INTS.items()})
        if self.nparts():
            out.update({k: self.coef(k) for k in COEF})
        return out

    def push(self):
        self.call("cuda_dom_push")
        self.call("cuda_part_push")

    def pull(self):
        self.call("cuda_dom_pull")
        self.call("cuda_part_pull")
        if self.devflags:
            self.pull_flags()

    devflags = None

    def pull_flags(self):
        """flag_u, flag_v, flag_w from the device through the reference's own
        device pointers (its cuda_part_pull copies them only when built
        with -DDDEBUG, src/cuda_particle.cu:282-291)"""
        for k in ("flag_u", "flag_v", "flag_w"):
            dev = C.POINTER(C.c_void_p).in_dll(self.lib, "_" + k)[0]
            host = self.arr(k, INTS[k], C.c_int)
            rc = self.devflags.cudaMemcpy(host.ctypes.data_as(C.c_void_p), C.c_void_p(dev),
                                          C.c_size_t(host.nbytes), 2)
            assert rc == 0, ("cudaMemcpy", k, rc)


def part_table(side):
    """the compared particle members as a dict of arrays"""
    recs = side.parts()
    out = {}
    for name, ctype in abi.PartStruct._fields_:
        if name in PSKIP:
            continue
        if name == "cage":
            for cn, _ in abi.CageStruct._fields_:
                out["cage." + cn] = np.array([getattr(q.cage, cn) for q in recs])
        elif hasattr(ctype, "_length_"):
            out[name] = np.array([list(getattr(q, name)) for q in recs])
        else:
            out[name] = np.array([getattr(q, name) for q in recs])
    return out


def copy_state(ref, ours):
    """the reference's host state into this library's host arrays"""
    ra, oa = ref.arrays(), ours.arrays()
    for k in ra:
        if ra[k].size and oa[k].size:
            oa[k][:] = ra[k]
    n = ref.nparts()
    if n:
        C.memmove(C.addressof(ours.parts()), C.addressof(ref.parts()),
                  n * C.sizeof(abi.PartStruct))
    for k in SCAL:
        ours.scalar(k).value = ref.scalar(k).value


GRIDS = dict(FACE, **CELL, **INTS)


def where(side, name, idx):
    """(i, j, k) of ghosted index idx in the array's grid"""
    g = getattr(side.dom, GRIDS[name])
    return [int(idx % g.s1b), int(idx // g.s1b % g.jnb), int(idx // g.s2b)]


def compare(ref, ours, before, before_parts, parts=False):
    """per array: largest |ref - ours|, largest |ref|, kind, largest change
    the stage made on the reference side, and for integer arrays the first
    differing cells (i, j, k, ref, ours) and their count"""
    res = {}
    ra, oa = ref.arrays(), ours.arrays()
    for k in ra:
        a, b = ra[k], oa[k]
        if not a.size or not b.size:
            continue
        diff = np.abs(a.astype(np.float64) - b)
        e = {"d": float(diff.max()), "mag": float(np.abs(a).max()),
             "kind": "int" if a.dtype.kind == "i" else "real",
             "moved": float(np.abs(a.astype(np.float64) - before[k]).max())}
        if e["kind"] == "int" and e["d"] > 0:
            bad = np.nonzero(diff)[0]
            e["count"] = int(bad.size)
            e["where"] = [where(ref, k, q) + [int(a[q]), int(b[q])] for q in bad[:8]]
        res[k] = e
    if parts and ref.nparts():
        pa, pb = part_table(ref), part_table(ours)
        for k in pa:
            a, b = pa[k].astype(np.float64), pb[k].astype(np.float64)
            res["parts." + k] = {"d": float(np.max(np.abs(a - b))),
                                 "mag": float(np.max(np.abs(a))),
                                 "kind": "int" if pa[k].dtype.kind in "iu" else "real",
                                 "moved": float(np.max(np.abs(a - before_parts[k])))}
    return res


def dia_apply(A, off, x):
    """y = A x for the 13-diagonal matrix in CUSP's dia layout"""
    n = x.size
    y = np.zeros(n)
    for d, o in enumerate(off):
        lo, hi = max(0, -o), min(n, n - o)
        if lo < hi:
            y[lo:hi] += A[d, lo:hi] * x[lo + o:hi + o]
    return y


def pp_system(ref, ours):
    """This library's pressure solve (cuda_PP_bicgstab) against the system
    the reference's own kernels assemble from the same state: the relative
    residual of the library's phi in the reference's system, after the
    constant shift the mean removal applied (fitted by least squares), and
    the same for the starting phi (that the system is not trivial)."""
    copy_state(ref, ours)
    ref.push()
    ours.push()
    g = ours.dom.Gcc
    inner = (slice(g.ks, g.ke), slice(g.js, g.je), slice(getattr(g, "is"), g.ie))
    shape = (g.knb, g.jnb, g.inb)
    x0 = ours.arr("phi", "Gcc").reshape(shape)[inner].ravel().copy()
    ours.call("cuda_PP_bicgstab", C.c_int(0))
    ours.pull()
    x = ours.arr("phi", "Gcc").reshape(shape)[inner].ravel().copy()
    n = ref.call("refshim_pp_rows", restype=C.c_int)
    assert n == x.size, (n, x.size)
    off = (C.c_int * 13)()
    ref.call("refshim_pp_offsets", off)
    A = np.zeros((13, n))
    b = np.zeros(n)
    rc = ref.call("refshim_pp_system", A.ctypes.data_as(C.c_void_p),
                  b.ctypes.data_as(C.c_void_p), restype=C.c_int)
    assert rc == 0, ("refshim_pp_system", rc)
    a1 = dia_apply(A, list(off), np.ones(n))

    def rel(v):
        r = b - dia_apply(A, list(off), v)
        c = float(a1 @ r) / float(a1 @ a1) if float(a1 @ a1) > 0 else 0.0
        return float(np.linalg.norm(r - c * a1) / max(np.linalg.norm(b), 1e-300))

    st = abi.Stats()
    ours.lib.bbb_get_stats(C.byref(st))
    return {"rel_resid": rel(x), "rel_resid_start": rel(x0),
            "b_norm": float(np.linalg.norm(b)), "kind": "system",
            "iterations": st.pp_iters_last,
            "identity_rows": int(np.sum(A[6] == 1.0))}


def helm_system(ref, ours, comp):
    """This library's Crank-Nicolson Helmholtz solve (cuda_{u,v,w}star_
    helmholtz) against the system the reference's own kernels assemble from
    the same state: the relative residual of the library's u* in it."""
    copy_state(ref, ours)
    ref.push()
    ours.push()
    name, grid = (("u_star", "Gfx"), ("v_star", "Gfy"), ("w_star", "Gfz"))[comp]
    g = getattr(ours.dom, grid)
    inner = (slice(g.ks, g.ke), slice(g.js, g.je), slice(getattr(g, "is"), g.ie))
    shape = (g.knb, g.jnb, g.inb)
    ours.call("cuda_%sstar_helmholtz" % "uvw"[comp], C.c_int(0))
    ours.pull()
    x = ours.arr(name, grid).reshape(shape)[inner].ravel().copy()
    n = ref.call("refshim_helm_rows", C.c_int(comp), restype=C.c_int)
    assert n == x.size, (n, x.size)
    off = (C.c_int * 13)()
    ref.call("refshim_helm_offsets", C.c_int(comp), off)
    A = np.zeros((13, n))
    b = np.zeros(n)
    rc = ref.call("refshim_helm_system", C.c_int(comp), A.ctypes.data_as(C.c_void_p),
                  b.ctypes.data_as(C.c_void_p), restype=C.c_int)
    assert rc == 0, ("refshim_helm_system", rc)
    r = b - dia_apply(A, list(off), x)
    bn = max(float(np.linalg.norm(b)), 1e-300)
    st = abi.Stats()
    ours.lib.bbb_get_stats(C.byref(st))
    return {"rel_resid": float(np.linalg.norm(r)) / bn,
            "solution_vs_rhs": float(np.linalg.norm(x - b)) / bn,
            "b_norm": bn, "identity_rows": int(np.sum(A[6] == 1.0)),
            "cg_iterations": st.helm_iters_total}


def main():
    run, out = sys.argv[1], sys.argv[2]
    implicit = len(sys.argv) > 3 and sys.argv[3] == "implicit"
    lib = abi.load()
    reflib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_gpu_implicit.so"
                                 if implicit else "libref_gpu.so"),
                    mode=os.RTLD_LOCAL | getattr(os, "RTLD_DEEPBIND", 0))
    os.chdir(run)
    lib.bbb_set_exit_on_failure(0)
    # the library in the form of the reference build it is checked against
    opts = abi.Options()
    lib.bbb_default_options(C.byref(opts))
    opts.implicit = 1 if implicit else 0
    opts.contact_overrun = 1     # the reference's slot-12 contact accesses
    lib.bbb_set_options(C.byref(opts))
    ref, ours = Side(reflib), Side(lib)
    for path in ("/usr/local/cuda/lib64/libcudart.so.12", "libcudart.so.12"):
        try:
            ref.devflags = C.CDLL(path)
            break
        except OSError:
            continue
    ref.devflags.cudaMemcpy.restype = C.c_int
    reflib.domain_read_input()
    reflib.parts_read_input(0)
    for f in ("domain_init", "parts_init", "binDom_init"):
        getattr(reflib, f).restype = C.c_int
        assert getattr(reflib, f)() == 0, f
    assert lib.bbb_read_input(b"input") == 0
    assert lib.bbb_domain_init() == 0
    assert lib.bbb_parts_init() == 0

    # the same seeded fields on both sides (ghost layers included)
    rng = np.random.default_rng(2024)
    for k, a in ref.arrays().items():
        if a.dtype.kind == "f":
            a[:] = 0.05 * rng.standard_normal(a.size)
        else:                       # fluid everywhere until the cages are built
            a[:] = -1 if k == "phase" else 1
    recs = ref.parts()
    for q in recs:
        q.u, q.v, q.w = 0.01 * rng.standard_normal(3)
        q.ox, q.oy, q.oz = 0.01 * rng.standard_normal(3)
    for k, v in (("dt", 0.01), ("dt0", 0.01), ("ttime", 0.5)):
        ref.scalar(k).value = v
    copy_state(ref, ours)

    for s in (ref, ours):
        s.call("cuda_dom_malloc")
        s.call("cuda_part_malloc")
        s.push()
    res = {}

    def stage(name, calls, parts=False, ret=None):
        copy_state(ref, ours)
        ref.push()
        ours.push()
        before = {k: a.astype(np.float64) for k, a in ref.arrays().items()}
        before_parts = {k: v.astype(np.float64) for k, v in part_table(ref).items()}
        got = []
        for s in (ref, ours):
            val = None
            for c in calls:
                rt = C.c_double if c == ret else None
                v = s.call(c, restype=rt)
                if c == ret:
                    val = v
            got.append(val)
            s.pull()
        r = compare(ref, ours, before, before_parts, parts=parts)
        if ret:
            r["return." + ret] = {"d": abs(got[0] - got[1]), "mag": abs(got[0]),
                                  "kind": "real"}
        res[name] = r
        assert lib.bbb_last_status() == 0, (name, lib.bbb_last_status())

    # src/bluebottle.c:603-708, the explicit step without the two solves
    stage("build_cages", ["cuda_build_cages"], parts=True)
    stage("dom_BC", ["cuda_dom_BC"])
    # the forcing fields live on the device only: both sides compute them
    # from the same clock and ramps (src/cuda_bluebottle.cu:3674), then the
    # right-hand sides below use them
    for s in (ref, ours):
        f = s.lib.cuda_compute_forcing
        f.restype = None
        f(C.byref(C.c_double.in_dll(s.lib, "pid_int")),
          C.byref(C.c_double.in_dll(s.lib, "pid_back")),
          C.c_double(C.c_double.in_dll(s.lib, "Kp").value),
          C.c_double(C.c_double.in_dll(s.lib, "Ki").value),
          C.c_double(C.c_double.in_dll(s.lib, "Kd").value))
    if not implicit:
        stage("U_star_2", ["cuda_U_star_2"])
    for comp in range(3):
        res["helmholtz_%s" % "uvw"[comp]] = helm_system(ref, ours, comp)
    stage("part_BC_star", ["cuda_part_BC_star", "cuda_dom_BC_star"])
    stage("solvability", ["cuda_solvability"])
    res["PP_system"] = pp_system(ref, ours)
    stage("project", ["cuda_dom_BC_phi", "cuda_project"])
    stage("part_BC", ["cuda_part_BC", "cuda_dom_BC"])
    stage("update_p", ["cuda_update_p"])
    stage("part_p_fill", ["cuda_part_BC", "cuda_part_p_fill", "cuda_dom_BC_p"])
    stage("move_parts_sub", ["cuda_move_parts_sub"], parts=True)
    stage("Lamb", ["cuda_Lamb", "cuda_lamb_err"], parts=True, ret="cuda_lamb_err")
    stage("move_parts", ["cuda_move_parts"], parts=True)
    stage("parts_internal", ["cuda_parts_internal", "cuda_dom_BC"])
    stage("store", ["cuda_store_u", "cuda_store_coeffs"], parts=True)
    stage("find_dt", ["cuda_find_dt"], ret="cuda_find_dt")
    stage("energy", ["cuda_compute_energy"], ret="cuda_compute_energy")
    for s in (ref, ours):
        s.call("cuda_part_free")
        s.call("cuda_dom_free")
    with open(out, "w") as fh:
        json.dump(res, fh)


if __name__ == "__main__":
    main()
