"""Host-side driver over the C ABI: the reference's set-up sequence and time
loop (src/bluebottle.c:415-708) plus access to the host arrays.

The library keeps the reference's process-global state, so one Sim is live
at a time.
"""
import ctypes as C
import os
import tempfile

import numpy as np

from . import abi

HOST_ARRAYS_CC = ("p0", "p", "phi")
HOST_ARRAYS_FACE = {"u": "Gfx", "u0": "Gfx", "u_star": "Gfx", "conv_u": "Gfx",
                    "conv0_u": "Gfx", "diff_u": "Gfx", "diff0_u": "Gfx",
                    "v": "Gfy", "v0": "Gfy", "v_star": "Gfy", "conv_v": "Gfy",
                    "conv0_v": "Gfy", "diff_v": "Gfy", "diff0_v": "Gfy",
                    "w": "Gfz", "w0": "Gfz", "w_star": "Gfz", "conv_w": "Gfz",
                    "conv0_w": "Gfz", "diff_w": "Gfz", "diff0_w": "Gfz"}
INT_ARRAYS = {"phase": "Gcc", "phase_shell": "Gcc", "flag_u": "Gfx",
              "flag_v": "Gfy", "flag_w": "Gfz"}
COEF_NAMES = ("pnm_re pnm_im phinm_re phinm_im chinm_re chinm_im "
              "pnm_re0 pnm_im0 phinm_re0 phinm_im0 chinm_re0 chinm_im0 "
              "pnm_re00 pnm_im00 phinm_re00 phinm_im00 chinm_re00 "
              "chinm_im00").split()
SCALARS_R = ("dt dt0 ttime rho_f nu mu CFL pp_residual lamb_residual "
             "lamb_relax lamb_cut vel_tDelay p_tDelay g_tDelay duration "
             "interactionLengthRatio Kp Ki Kd pid_int pid_back").split()
SCALARS_I = ("pp_max_iter lamb_max_iter out_plane stepnum init_cond nparts "
             "coeff_stride nsubdom").split()


class BBBError(RuntimeError):
    pass


class Sim:
    """One simulation driven through libbbb200.so.

    workload: a bluebottle_b200.configs.Workload, or None with `input_dir`
    pointing at a directory holding flow.config / part.config.
    """

    def __init__(self, workload=None, input_dir=None, options=None,
                 exit_on_failure=False):
        self.lib = abi.load()
        lib = self.lib
        lib.bbb_set_exit_on_failure(1 if exit_on_failure else 0)
        lib.bbb_clear_status()
        self._tmp = None
        if workload is not None and input_dir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="bbb_")
            input_dir = workload.write(self._tmp.name)
        opts = abi.Options()
        lib.bbb_default_options(C.byref(opts))
        merged = dict(workload.options) if workload is not None else {}
        merged.update(options or {})
        for k, v in merged.items():
            setattr(opts, k, v)
        lib.bbb_set_options(C.byref(opts))
        self.options = opts
        self._check(lib.bbb_read_input(input_dir.encode()), "read_input")
        self._check(lib.bbb_domain_init(), "domain_init")
        if workload is not None and workload.taylor_green:
            lib.bbb_init_taylor_green(workload.taylor_green)
        if workload is not None and workload.npart > 0:
            self._check(lib.bbb_seed_particles(
                workload.npart, workload.a, workload.gap, workload.rho_p,
                workload.order, workload.rsr, workload.seed), "seed")
        self._check(lib.bbb_parts_init(), "parts_init")
        self.prepared = False

    def _check(self, rc, where):
        if rc != 0:
            msg = self.lib.bbb_status_string(rc).decode()
            raise BBBError("%s: %s" % (where, msg))

    # -------------------------------------------------------- host state
    @property
    def dom(self):
        return abi.DomStruct.in_dll(self.lib, "Dom")

    def scalar(self, name):
        t = C.c_int if name in SCALARS_I else C.c_double
        return t.in_dll(self.lib, name).value

    def set_scalar(self, name, value):
        t = C.c_int if name in SCALARS_I else C.c_double
        t.in_dll(self.lib, name).value = value

    @property
    def bc(self):
        return abi.BCStruct.in_dll(self.lib, "bc")

    @property
    def g(self):
        return abi.GStruct.in_dll(self.lib, "g")

    @property
    def gradP(self):
        return abi.GStruct.in_dll(self.lib, "gradP")

    @property
    def nparts(self):
        return self.scalar("nparts")

    def array(self, name):
        d = self.dom
        if name in HOST_ARRAYS_CC:
            return abi.host_array(self.lib, name, d.Gcc.s3b)
        if name in HOST_ARRAYS_FACE:
            return abi.host_array(self.lib, name, getattr(d, HOST_ARRAYS_FACE[name]).s3b)
        if name in INT_ARRAYS:
            return abi.host_array(self.lib, name, getattr(d, INT_ARRAYS[name]).s3b,
                                  C.c_int)
        if name in COEF_NAMES:
            return abi.host_array(self.lib, name,
                                  self.nparts * self.scalar("coeff_stride"))
        raise KeyError(name)

    def parts(self):
        n = self.nparts
        ptr = C.POINTER(abi.PartStruct).in_dll(self.lib, "parts")
        if n <= 0 or not ptr:
            return []
        return (abi.PartStruct * n).from_address(C.addressof(ptr.contents))

    # -------------------------------------------------------- device
    def prepare(self):
        self._check(self.lib.bbb_prepare(), "prepare")
        self.prepared = True

    def step(self):
        rc = self.lib.bbb_step()
        if rc != 0:
            raise BBBError("step: %s" % self.lib.bbb_status_string(rc).decode())

    def stats(self):
        st = abi.Stats()
        self.lib.bbb_get_stats(C.byref(st))
        return st

    def pull(self):
        self.lib.cuda_dom_pull()
        self.lib.cuda_part_pull()

    # -------------------------------------------------------- restart
    def out_restart(self, path):
        """Write the reference's restart file from the host copies (pull
        first when the simulation has run on the device)."""
        self._check(self.lib.bbb_out_restart(os.fsencode(path)), "out_restart")

    def write_part_config(self, path):
        """Write the particle list as the reference's part.config."""
        self._check(self.lib.bbb_write_part_config(os.fsencode(path)),
                    "write_part_config")

    def in_restart(self, path):
        """Read a restart file into the host copies (push, or prepare,
        afterwards to run from it)."""
        self._check(self.lib.bbb_in_restart(os.fsencode(path)), "in_restart")

    def push(self):
        self.lib.cuda_dom_push()
        self.lib.cuda_part_push()

    def divergence(self):
        mx, l2 = C.c_double(), C.c_double()
        self.lib.bbb_divergence(C.byref(mx), C.byref(l2))
        return mx.value, l2.value

    def energy(self):
        return self.lib.cuda_compute_energy()

    def status(self):
        return self.lib.bbb_last_status()

    def close(self):
        if self.prepared:
            self.lib.bbb_release()
            self.prepared = False
        self.lib.bbb_host_free()
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def interior(a, G):
    """Interior block of a ghosted array on grid_info G as (k, j, i)."""
    a3 = np.asarray(a).reshape(G.knb, G.jnb, G.inb)
    i0, i1 = getattr(G, "is"), G.ie
    return a3[G.ks:G.ke, G.js:G.je, i0:i1]
