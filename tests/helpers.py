import numpy as np

from bluebottle_b200 import interior


def rel_err(a, b):
    """max |a - b| / max |b| (absolute when b is identically zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b)) if b.size else 0.0
    num = np.max(np.abs(a - b)) if b.size else 0.0
    return num / den if den > 0 else num


FIELD_GRIDS = {"u": "Gfx", "v": "Gfy", "w": "Gfz", "p": "Gcc", "phi": "Gcc",
               "u_star": "Gfx", "v_star": "Gfy", "w_star": "Gfz",
               "conv_u": "Gfx", "conv_v": "Gfy", "conv_w": "Gfz",
               "u0": "Gfx", "v0": "Gfy", "w0": "Gfz", "p0": "Gcc",
               "phase": "Gcc", "phase_shell": "Gcc", "flag_u": "Gfx",
               "flag_v": "Gfy", "flag_w": "Gfz"}


def field_interior(dom, name, arr):
    return interior(arr, getattr(dom, FIELD_GRIDS[name]))
