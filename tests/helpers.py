import os

import numpy as np

from bluebottle_b200 import interior

# the reference checkout the reference-built checkers compile from (only
# where it exists; the tests that need it skip otherwise)
REF_ROOT = os.environ.get("BLUEBOTTLE_REF", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "src")


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


def grid_xyz(dom, G, offs):
    """Coordinates of every point (ghosts included) of grid G, x fastest;
    offs = index offsets of the point from the cell's lower corner
    (1.0 for a face position, 0.5 for a centre, as src/cuda_testing.cu)."""
    i = np.arange(G.isb, G.ieb)
    j = np.arange(G.jsb, G.jeb)
    k = np.arange(G.ksb, G.keb)
    x = (i - offs[0]) * dom.dx + dom.xs
    y = (j - offs[1]) * dom.dy + dom.ys
    z = (k - offs[2]) * dom.dz + dom.zs
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return X, Y, Z


def stokes_case(tmp_path, n=48, L=3.0, nu=1.0):
    """One sphere of radius 1 at the centre of the periodic box [-L, L]^3
    (the set-up of cuda_lamb_test, src/cuda_testing.cu:1836)."""
    import os
    from bluebottle_b200 import Sim, configs
    d = str(tmp_path)
    configs.write_flow_config(os.path.join(d, "flow.config"), n=(n, n, n),
                              lo=(-L,) * 3, hi=(L,) * 3, nu=nu, rho_f=1.0,
                              lamb_max_iter=1)
    configs.write_part_config(os.path.join(d, "part.config"),
                              [dict(r=1.0, x=0.0, y=0.0, z=0.0, order=4)])
    return Sim(input_dir=d)


def stokes_fields(sim, W=0.01, a=1.0):
    """Stokes flow past a fixed sphere, uniform velocity (0, 0, W) far away:
    p = -3/2 mu a (U.r)/r^3 and the classical velocity field, evaluated at
    every ghosted point of each grid (src/cuda_testing.cu:1907-1989)."""
    d = sim.dom
    out = {}
    X, Y, Z = grid_xyz(d, d.Gcc, (0.5, 0.5, 0.5))
    r = np.sqrt(X * X + Y * Y + Z * Z)
    out["p"] = (-1.5 * (W * Z / r) * a / r / r).ravel()
    for nm, G, offs, comp in (("u", d.Gfx, (1.0, 0.5, 0.5), 0),
                              ("v", d.Gfy, (0.5, 1.0, 0.5), 1),
                              ("w", d.Gfz, (0.5, 0.5, 1.0), 2)):
        X, Y, Z = grid_xyz(d, G, offs)
        r = np.sqrt(X * X + Y * Y + Z * Z)
        ud = W * Z / r
        xc = (X, Y, Z)[comp] / r
        Uc = W if comp == 2 else 0.0
        val = (-0.75 * a / r * (Uc + ud * xc)
               - 0.25 * a ** 3 / r ** 3 * (Uc - 3.0 * ud * xc) + Uc)
        out[nm] = val.ravel()
    return out
