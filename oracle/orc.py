"""ctypes wrapper of the CPU FP64 oracle (liborc.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the result to check against.  Nothing in bluebottle_b200
imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from bluebottle_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liborc.so")


class OrcParams(C.Structure):
    _fields_ = [("rho_f", C.c_double), ("nu", C.c_double), ("mu", C.c_double),
                ("dt", C.c_double), ("dt0", C.c_double), ("ttime", C.c_double),
                ("CFL", C.c_double), ("pp_max_iter", C.c_int),
                ("pp_residual", C.c_double), ("lamb_max_iter", C.c_int),
                ("lamb_residual", C.c_double), ("lamb_relax", C.c_double),
                ("lamb_cut", C.c_double), ("out_plane", C.c_int),
                ("implicit", C.c_int), ("fixed_dt", C.c_double),
                ("vel_tDelay", C.c_double), ("p_tDelay", C.c_double),
                ("g_tDelay", C.c_double), ("Kp", C.c_double),
                ("Ki", C.c_double), ("Kd", C.c_double),
                ("pid_int", C.c_double), ("pid_back", C.c_double),
                ("interactionLengthRatio", C.c_double),
                ("bc", abi.BCStruct), ("g", abi.GStruct),
                ("gradP", abi.GStruct), ("stepnum", C.c_int),
                ("contact_overrun", C.c_int)]


_lib = None


def build():
    srcs = [os.path.join(HERE, f) for f in ("orc_fluid.c", "orc_part.c", "orc.h")]
    if (not os.path.exists(LIB)) or any(os.path.getmtime(s) > os.path.getmtime(LIB)
                                        for s in srcs):
        subprocess.run(["make", "-s", "-C", HERE, "liborc.so"], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    lib = C.CDLL(LIB)
    vp = C.c_void_p
    lib.orc_create.restype = vp
    lib.orc_create.argtypes = [C.POINTER(abi.DomStruct), C.c_int, C.c_int]
    lib.orc_destroy.argtypes = [vp]
    lib.orc_field.restype = vp
    lib.orc_field.argtypes = [vp, C.c_char_p, C.POINTER(C.c_long)]
    lib.orc_params_ptr.restype = C.POINTER(OrcParams)
    lib.orc_params_ptr.argtypes = [vp]
    lib.orc_get_stats.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    lib.orc_set_threads.restype = C.c_int
    lib.orc_set_threads.argtypes = [C.c_int]
    for name in ("orc_compute_forcing", "orc_compute_vel_BC", "orc_U_star_2",
                 "orc_solvability", "orc_PP_rhs", "orc_PP_bicgstab",
                 "orc_project", "orc_update_p", "orc_store_u",
                 "orc_build_cages", "orc_part_BC_p", "orc_part_p_fill",
                 "orc_parts_internal", "orc_Lamb", "orc_store_coeffs",
                 "orc_move_parts_sub", "orc_move_parts"):
        getattr(lib, name).argtypes = [vp]
    for name in ("orc_dom_BC", "orc_star_rhs", "orc_star_helmholtz",
                 "orc_part_BC"):
        getattr(lib, name).argtypes = [vp, C.c_int]
    for name in ("orc_find_dt", "orc_lamb_err", "orc_compute_energy"):
        getattr(lib, name).argtypes = [vp]
        getattr(lib, name).restype = C.c_double
    lib.orc_step.argtypes = [vp]
    lib.orc_step.restype = C.c_int
    dp = C.POINTER(C.c_double)
    lib.orc_poisson_apply.argtypes = [vp, dp, dp]
    lib.orc_poisson_solve.argtypes = [vp, dp, dp, C.c_double, C.c_int, dp]
    lib.orc_poisson_solve.restype = C.c_int
    lib.orc_divergence.argtypes = [vp, dp, dp, dp, dp, dp]
    _lib = lib
    return lib


INT_FIELDS = ("phase", "phase_shell", "flag_u", "flag_v", "flag_w")

REF_DIR = os.path.join(HERE, "_ref")


def reference_host_lib(implicit=True):
    """Path of the reference's own host set-up code built by oracle/ref.mk
    (src/domain.c, src/particle.c, src/rng.c; the -DIMPLICIT build for the
    Crank-Nicolson program), or None when it has not been built."""
    p = os.path.join(REF_DIR, "libref_host_implicit.so" if implicit
                     else "libref_host.so")
    return p if os.path.exists(p) else None


def reference_setup(run_dir, implicit=True):
    """Run the reference's host set-up in run_dir (which holds
    input/flow.config and input/part.config): domain_read_input,
    parts_read_input, domain_init, parts_init (src/bluebottle.c:415-431).
    Returns the loaded library, whose globals hold the state."""
    path = reference_host_lib(implicit)
    if path is None:
        raise FileNotFoundError("oracle/_ref/libref_host*.so is not built")
    ref = C.CDLL(path, mode=os.RTLD_LOCAL | getattr(os, "RTLD_DEEPBIND", 0))
    ref.domain_init.restype = C.c_int
    ref.parts_init.restype = C.c_int
    cwd = os.getcwd()
    os.chdir(run_dir)
    try:
        ref.domain_read_input()
        ref.parts_read_input(0)
        if ref.domain_init() != 0 or ref.parts_init() != 0:
            raise RuntimeError("the reference's domain_init/parts_init failed")
    finally:
        os.chdir(cwd)
    return ref


class Oracle:
    """FP64 CPU state mirroring the reference's host arrays."""

    def __init__(self, dom, nparts, coeff_stride):
        self.lib = load()
        self.dom = abi.DomStruct.from_buffer_copy(dom)
        self.st = self.lib.orc_create(C.byref(self.dom), nparts, coeff_stride)
        self.nparts = nparts
        self.coeff_stride = coeff_stride

    @property
    def P(self):
        return self.lib.orc_params_ptr(self.st).contents

    def field(self, name):
        n = C.c_long()
        ptr = self.lib.orc_field(self.st, name.encode(), C.byref(n))
        if not ptr:
            raise KeyError(name)
        if name == "parts":
            return (abi.PartStruct * n.value).from_address(ptr) if n.value else []
        ct = C.c_int if name in INT_FIELDS else C.c_double
        if n.value == 0:
            return np.zeros(0)
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(n.value,))

    def stats(self):
        iv = (C.c_int * 8)()
        rv = (C.c_double * 5)()
        self.lib.orc_get_stats(self.st, iv, rv)
        return dict(pp_iters=iv[0], pp_converged=iv[1], pp_solves=iv[2],
                    pp_iters_total=iv[3], cg_iters=list(iv[4:7]),
                    lamb_iters=iv[7], pp_resid=rv[0], lamb_err=rv[1],
                    cg_resid=list(rv[2:5]))

    REAL_PARAMS = ("rho_f", "nu", "mu", "dt", "dt0", "ttime", "CFL",
                   "pp_residual", "lamb_residual", "lamb_relax", "lamb_cut",
                   "vel_tDelay", "p_tDelay", "g_tDelay", "Kp", "Ki", "Kd",
                   "pid_int", "pid_back", "interactionLengthRatio")
    INT_PARAMS = ("pp_max_iter", "lamb_max_iter", "out_plane", "stepnum")
    FIELD_NAMES = ("p0", "p", "phi", "u", "v", "w", "u0", "v0", "w0",
                   "u_star", "v_star", "w_star", "conv_u", "conv_v",
                   "conv_w", "conv0_u", "conv0_v", "conv0_w", "diff_u",
                   "diff_v", "diff_w", "diff0_u", "diff0_v", "diff0_w")

    @classmethod
    def _from_host(cls, dom, nparts, coeff_stride, scalar, array, bc, g, gradP,
                   parts_addr, implicit, fixed_dt, lamb_override, prepare,
                   contact_overrun=0):
        o = cls(dom, nparts, coeff_stride)
        P = o.P
        for k in cls.REAL_PARAMS + cls.INT_PARAMS:
            setattr(P, k, scalar(k))
        P.implicit = implicit
        P.fixed_dt = fixed_dt
        P.contact_overrun = contact_overrun
        if lamb_override > 0:
            P.lamb_max_iter = lamb_override
        C.memmove(C.byref(P.bc), C.byref(bc), C.sizeof(abi.BCStruct))
        C.memmove(C.byref(P.g), C.byref(g), C.sizeof(abi.GStruct))
        C.memmove(C.byref(P.gradP), C.byref(gradP), C.sizeof(abi.GStruct))
        for name in cls.FIELD_NAMES:
            a = array(name, o.field(name).size)
            if a is not None:
                o.field(name)[:] = a
        if nparts > 0:
            dst = o.field("parts")
            C.memmove(C.addressof(dst), parts_addr,
                      C.sizeof(abi.PartStruct) * nparts)
            from bluebottle_b200.sim import COEF_NAMES
            for name in COEF_NAMES:
                a = array(name, o.field(name).size)
                if a is not None:
                    o.field(name)[:] = a
        if prepare:
            o.prepare()
        return o

    @classmethod
    def from_sim(cls, sim, prepare=True):
        """Copy a Sim's host state after its host initialisation (before or
        without its device set-up) and, optionally, run the reference's
        set-up sequence (src/bluebottle.c:528-543) on the CPU."""
        n = sim.nparts
        addr = C.addressof(sim.parts()) if n > 0 else 0
        return cls._from_host(
            sim.dom, n, sim.scalar("coeff_stride"), sim.scalar,
            lambda name, size: sim.array(name), sim.bc, sim.g, sim.gradP,
            addr, sim.options.implicit, sim.options.fixed_dt,
            sim.options.lamb_max_iter_override, prepare,
            sim.options.contact_overrun)

    @classmethod
    def from_reference(cls, ref, implicit=1, fixed_dt=0.0, lamb_override=0,
                       prepare=True):
        """Copy the host state the reference's own set-up left in `ref`
        (a library from reference_setup): its Dom, boundary conditions,
        scalars, initial fields, particle records and Lamb coefficients."""
        real_names = set(cls.REAL_PARAMS)

        def scalar(name):
            t = C.c_double if name in real_names else C.c_int
            return t.in_dll(ref, name).value

        def array(name, size):
            ptr = C.POINTER(C.c_double).in_dll(ref, name)
            if not ptr:
                return None       # not allocated by this build (-DIMPLICIT)
            return np.ctypeslib.as_array(ptr, shape=(size,))

        n = C.c_int.in_dll(ref, "nparts").value
        addr = 0
        if n > 0:
            addr = C.addressof(C.POINTER(abi.PartStruct).in_dll(ref, "parts").contents)
        return cls._from_host(
            abi.DomStruct.in_dll(ref, "Dom"), n,
            C.c_int.in_dll(ref, "coeff_stride").value, scalar, array,
            abi.BCStruct.in_dll(ref, "bc"), abi.GStruct.in_dll(ref, "g"),
            abi.GStruct.in_dll(ref, "gradP"), addr, implicit, fixed_dt,
            lamb_override, prepare)

    def prepare(self):
        lib, st = self.lib, self.st
        lib.orc_build_cages(st)
        dt = lib.orc_find_dt(st)
        self.P.dt = self.P.fixed_dt if self.P.fixed_dt > 0 else dt
        if self.nparts > 0:
            lib.orc_part_BC(st, 0)
        lib.orc_dom_BC(st, 0)
        lib.orc_parts_internal(st)
        lib.orc_dom_BC(st, 0)

    def step(self):
        return self.lib.orc_step(self.st)

    def energy(self):
        return self.lib.orc_compute_energy(self.st)

    def divergence(self):
        mx, l2 = C.c_double(), C.c_double()
        dp = C.POINTER(C.c_double)
        self.lib.orc_divergence(self.st, self.field("u").ctypes.data_as(dp),
                                self.field("v").ctypes.data_as(dp),
                                self.field("w").ctypes.data_as(dp),
                                C.byref(mx), C.byref(l2))
        return mx.value, l2.value

    def close(self):
        if self.st:
            self.lib.orc_destroy(self.st)
            self.st = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
