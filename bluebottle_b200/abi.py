"""ctypes view of the libbbb200.so C ABI (include/bluebottle_b200.h).

The structs mirror include/bluebottle_b200_types.h, which keeps the
reference's member order (src/domain.h, src/bluebottle.h, src/particle.h).
Loading fails loudly when the library has not been built: there is no CPU
fallback for anything in this package.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbbb200.so")

_GRID_NAMES = ("is ie in isb ieb inb js je jn jsb jeb jnb ks ke kn ksb keb knb "
               "s1 s1b s2 s2b s3 s3b").split()


class GridInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in _GRID_NAMES] + \
               [("_" + n, C.c_int) for n in _GRID_NAMES]


class DomStruct(C.Structure):
    _fields_ = [("Gcc", GridInfo), ("Gfx", GridInfo), ("Gfy", GridInfo),
                ("Gfz", GridInfo),
                ("xs", C.c_double), ("xe", C.c_double), ("xl", C.c_double),
                ("xn", C.c_int), ("dx", C.c_double),
                ("ys", C.c_double), ("ye", C.c_double), ("yl", C.c_double),
                ("yn", C.c_int), ("dy", C.c_double),
                ("zs", C.c_double), ("ze", C.c_double), ("zl", C.c_double),
                ("zn", C.c_int), ("dz", C.c_double),
                ("E", C.c_int), ("W", C.c_int), ("N", C.c_int), ("S", C.c_int),
                ("T", C.c_int), ("B", C.c_int)]


class GStruct(C.Structure):
    _fields_ = [(n, C.c_double) for n in "x xm xa y ym ya z zm za".split()]


GradPStruct = GStruct


def _bc_fields():
    f = []
    for face in "WESNBT":
        f += [("p" + face, C.c_int), ("p" + face + "D", C.c_double)]
    for comp in "uvw":
        for face in "WESNBT":
            f += [(comp + face, C.c_int), (comp + face + "Dm", C.c_double),
                  (comp + face + "D", C.c_double),
                  (comp + face + "Da", C.c_double)]
    f += [("ds" + face, C.c_double) for face in "WESNBT"]
    return f


class BCStruct(C.Structure):
    _fields_ = _bc_fields()


class CageStruct(C.Structure):
    _fields_ = [(n, C.c_int) for n in
                "cx cy cz is ibs ie ibe in js jbs je jbe jn ks kbs ke kbe kn".split()]


_PART_REALS1 = ("r x y z x0 y0 z0 u v w u0 v0 w0 udot vdot wdot udot0 vdot0 "
                "wdot0 axx axy axz ayx ayy ayz azx azy azz ox oy oz ox0 oy0 "
                "oz0 oxdot oydot ozdot oxdot0 oydot0 ozdot0 Fx Fy Fz Lx Ly Lz "
                "aFx aFy aFz aLx aLy aLz kFx kFy kFz iFx iFy iFz iLx iLy "
                "iLz").split()


class PartStruct(C.Structure):
    _fields_ = [(n, C.c_double) for n in _PART_REALS1] + [
        ("nodes", C.c_int * 26), ("rho", C.c_double), ("E", C.c_double),
        ("sigma", C.c_double), ("cage", CageStruct), ("order", C.c_int),
        ("rs", C.c_double), ("ncoeff", C.c_int), ("spring_k", C.c_double),
        ("spring_x", C.c_double), ("spring_y", C.c_double),
        ("spring_z", C.c_double), ("spring_l", C.c_double),
        ("translating", C.c_int), ("rotating", C.c_int), ("bin", C.c_int),
        ("St", C.c_double * 12), ("iSt", C.c_int * 12),
        ("e_dry", C.c_double), ("coeff_fric", C.c_double)]


class Options(C.Structure):
    _fields_ = [("implicit", C.c_int), ("fixed_dt", C.c_double),
                ("precision", C.c_int), ("inner_tol", C.c_double),
                ("max_outer", C.c_int), ("learned_guess", C.c_int),
                ("record", C.c_int), ("gravity_balance", C.c_int),
                ("lamb_max_iter_override", C.c_int), ("verbose", C.c_int),
                ("reliable", C.c_int), ("contact_overrun", C.c_int),
                ("lamb_pp_tol", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("pp_solves", C.c_int), ("pp_iters_total", C.c_int),
                ("pp_iters_last", C.c_int), ("pp_resid_last", C.c_double),
                ("pp_outer_last", C.c_int), ("helm_iters_total", C.c_int),
                ("lamb_iters", C.c_int), ("lamb_err", C.c_double),
                ("guess_used", C.c_int), ("guess_r0", C.c_double),
                ("extrap_r0", C.c_double), ("guess_evaluated", C.c_int),
                ("guess_cost_ms", C.c_double), ("guess_benefit_ms", C.c_double),
                ("step_dt", C.c_double), ("cfl_adv", C.c_double),
                ("helm_solves", C.c_int), ("pp_iters_max", C.c_int),
                ("pp_iters_first", C.c_int)]


PERIODIC, DIRICHLET, NEUMANN, PRECURSOR = 0, 1, 2, 3
PREC_FP64, PREC_MIXED = 0, 1
STATUS = {0: "ok", 1: "cuda", 2: "not converged", 3: "config",
          4: "unsupported", 5: "state", 6: "diverged", 7: "too large",
          8: "non-finite"}

# every extern "C" function include/bluebottle_b200.h declares
DECLARED = """cuda_dom_malloc cuda_part_malloc cuda_dom_push cuda_part_push
cuda_dom_pull cuda_part_pull cuda_dom_free cuda_part_free cuda_compute_forcing
cuda_build_cages cuda_U_star_2 cuda_ustar_helmholtz cuda_vstar_helmholtz
cuda_wstar_helmholtz cuda_ustar_rhs cuda_vstar_rhs cuda_wstar_rhs cuda_PP_rhs
cuda_part_BC cuda_part_BC_star cuda_part_BC_p cuda_part_p_fill cuda_dom_BC
cuda_dom_BC_star cuda_dom_BC_phi cuda_dom_BC_p cuda_solvability
cuda_PP_bicgstab cuda_project cuda_update_p cuda_move_parts_sub
cuda_move_parts cuda_Lamb cuda_lamb_err cuda_parts_internal cuda_store_u
cuda_store_coeffs cuda_find_dt cuda_compute_energy cuda_div_U
cuda_dom_turb_planes_push cuda_dom_turb_planes_pull cuda_compute_turb_forcing
cuda_yank_turb_planes bbb_default_options bbb_set_options bbb_get_options
bbb_read_input bbb_domain_init bbb_parts_init bbb_seed_particles
bbb_write_part_config
bbb_init_taylor_green bbb_host_free bbb_out_restart bbb_in_restart
bbb_prepare bbb_release
bbb_set_record_dir bbb_step bbb_advance_clock bbb_get_stats bbb_last_status
bbb_status_string bbb_clear_status bbb_set_exit_on_failure bbb_device_count
bbb_divergence bbb_kernel_launches bbb_reset_kernel_launches
bbb_profile_enable bbb_profile_reset bbb_profile_get bbb_profile_get_pass
bbb_stage_layout
bbb_part_state_push
bbb_part_state_pull bbb_mark bbb_mark_elapsed bbb_PP_bicgstab_static
bbb_learn_enable bbb_learn_train bbb_learn_crops bbb_learn_param_count
bbb_learn_get_params bbb_learn_set_params bbb_learn_forward
bbb_learn_use_reference_conv bbb_learn_grad bbb_learn_gate_decide
bbb_learn_set_crops_per_step bbb_snapshot_start bbb_snapshot_finish
bbb_snapshot_busy""".split()

_lib = None


def load():
    """Load libbbb200.so once and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            "libbbb200.so is not built; run `python -m bluebottle_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH, mode=C.RTLD_GLOBAL)
    R = C.c_double
    for name in DECLARED:
        getattr(lib, name).restype = None
    for name in ("cuda_lamb_err", "cuda_find_dt", "cuda_compute_energy"):
        getattr(lib, name).restype = R
    for name in ("bbb_read_input", "bbb_domain_init", "bbb_parts_init",
                 "bbb_seed_particles", "bbb_step", "bbb_last_status",
                 "bbb_device_count", "bbb_prepare", "bbb_learn_enable",
                 "bbb_learn_crops", "bbb_learn_param_count",
                 "bbb_learn_get_params", "bbb_learn_set_params",
                 "bbb_learn_forward", "bbb_PP_bicgstab_static",
                 "bbb_learn_set_crops_per_step", "bbb_snapshot_start",
                 "bbb_snapshot_finish", "bbb_snapshot_busy",
                 "bbb_out_restart", "bbb_in_restart"):
        getattr(lib, name).restype = C.c_int
    lib.bbb_out_restart.argtypes = [C.c_char_p]
    lib.bbb_in_restart.argtypes = [C.c_char_p]
    lib.bbb_kernel_launches.restype = C.c_longlong
    lib.bbb_status_string.restype = C.c_char_p
    lib.bbb_read_input.argtypes = [C.c_char_p]
    lib.bbb_set_record_dir.argtypes = [C.c_char_p]
    lib.bbb_seed_particles.argtypes = [C.c_int, R, R, R, C.c_int, R,
                                       C.c_ulonglong]
    lib.bbb_init_taylor_green.argtypes = [R]
    lib.bbb_set_options.argtypes = [C.POINTER(Options)]
    lib.bbb_get_options.argtypes = [C.POINTER(Options)]
    lib.bbb_default_options.argtypes = [C.POINTER(Options)]
    lib.bbb_get_stats.argtypes = [C.POINTER(Stats)]
    lib.bbb_divergence.argtypes = [C.POINTER(R), C.POINTER(R)]
    lib.cuda_compute_forcing.argtypes = [C.POINTER(R), C.POINTER(R), R, R, R]
    lib.bbb_profile_enable.argtypes = [C.c_int]
    lib.bbb_mark.argtypes = [C.c_int]
    vp = C.c_void_p
    lib.bbb_PP_bicgstab_static.restype = C.c_int
    lib.bbb_PP_bicgstab_static.argtypes = [
        C.c_int, C.c_int, C.c_int, R, R, R, C.c_int, C.c_int, C.c_int,
        vp, vp, vp, vp, vp, vp, vp, R, R, R, C.c_int, vp,
        C.POINTER(C.c_int), C.POINTER(R), vp]
    lib.bbb_mark_elapsed.argtypes = [C.c_int, C.c_int]
    lib.bbb_mark_elapsed.restype = R
    lib.bbb_profile_get.argtypes = [C.POINTER(R), C.POINTER(C.c_longlong),
                                    C.POINTER(R)]
    lib.bbb_profile_get_pass.argtypes = [C.c_int, C.POINTER(R),
                                         C.POINTER(C.c_longlong), C.POINTER(R)]
    lib.bbb_stage_layout.restype = C.c_int
    lib.bbb_stage_layout.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int]
    lib.bbb_learn_enable.argtypes = [C.c_int]
    lib.bbb_learn_train.argtypes = [C.c_int, R]
    lib.bbb_learn_train.restype = R
    lib.bbb_learn_get_params.argtypes = [C.POINTER(C.c_float), C.c_int]
    lib.bbb_learn_set_params.argtypes = [C.POINTER(C.c_float), C.c_int]
    lib.bbb_learn_forward.argtypes = [C.c_int] * 6 + [vp, vp, C.c_int]
    lib.bbb_learn_use_reference_conv.argtypes = [C.c_int]
    lib.bbb_learn_gate_decide.argtypes = [R] * 5 + [C.POINTER(C.c_int), C.POINTER(R)]
    lib.bbb_learn_gate_decide.restype = C.c_int
    lib.bbb_write_part_config.argtypes = [C.c_char_p]
    lib.bbb_write_part_config.restype = C.c_int
    lib.bbb_learn_grad.argtypes = [C.c_int] * 5 + [vp, vp, C.POINTER(C.c_float)]
    lib.bbb_learn_grad.restype = R
    for name in ("cuda_ustar_helmholtz", "cuda_vstar_helmholtz",
                 "cuda_wstar_helmholtz", "cuda_PP_bicgstab", "cuda_PP_rhs",
                 "cuda_part_BC_p", "cuda_ustar_rhs", "cuda_vstar_rhs",
                 "cuda_wstar_rhs"):
        getattr(lib, name).argtypes = [C.c_int]
    _lib = lib
    return lib


def glob(lib, ctype, name):
    """A reference global of libbbb200.so as a ctypes object."""
    return ctype.in_dll(lib, name)


def host_array(lib, name, count, ctype=C.c_double):
    """numpy view of a host array held in a pointer global."""
    ptr = C.POINTER(ctype).in_dll(lib, name)
    if not ptr or count <= 0:
        return np.zeros(0, dtype=np.float64 if ctype is C.c_double else np.int32)
    return np.ctypeslib.as_array(ptr, shape=(count,))
