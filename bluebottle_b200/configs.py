"""Writers for the reference's input files and the benchmark workloads.

flow.config and part.config are written in the strict-order format the
reference's readers expect (src/domain.c:30-730, src/particle.c:79-159), so
the same directory also runs under the reference.  Settings the reference
has no key for (fixed dt, Taylor-Green start, seeded packs, precision form)
are returned separately as build-side options.
"""
import os
from dataclasses import dataclass, field


def _fmt(v):
    return repr(float(v))


def write_flow_config(path, *, n=(32, 32, 32), lo=(0.0, 0.0, 0.0),
                      hi=(1.0, 1.0, 1.0), rho_f=1.0, nu=1.0, duration=1.0,
                      CFL=0.5, pp_max_iter=2000, pp_residual=1e-8,
                      lamb_max_iter=25, lamb_residual=1e-2, lamb_relax=1.0,
                      lamb_cut=1e-4, periodic=(True, True, True),
                      init_cond="QUIESCENT", out_plane="HOMOGENEOUS",
                      gradP=(0.0, 0.0, 0.0), g=(0.0, 0.0, 0.0),
                      walls_dirichlet=None):
    """Write flow.config.  Non-periodic axes get no-slip Dirichlet walls and
    Neumann pressure unless `walls_dirichlet` says otherwise."""
    L = []
    L.append("DOMAIN")
    for ax, nm in enumerate("XYZ"):
        L.append("(%ss, %se, %sn) %s %s %d" % (nm, nm, nm, _fmt(lo[ax]),
                                               _fmt(hi[ax]), n[ax]))
    L.append("")
    L.append("GPU DOMAIN DECOMPOSITION")
    L.append("DEV RANGE 0 0")
    L.append("n 1")
    for ax, nm in enumerate("XYZ"):
        L.append("(%ss, %se, %sn) %s %s %d" % (nm, nm, nm, _fmt(lo[ax]),
                                               _fmt(hi[ax]), n[ax]))
    L.append("E -1 W -1 N -1 S -1 T -1 B -1")
    L.append("")
    L.append("PHYSICAL PARAMETERS")
    L.append("rho_f %s" % _fmt(rho_f))
    L.append("nu %s" % _fmt(nu))
    L.append("")
    L.append("SIMULATION PARAMETERS")
    L.append("duration %s" % _fmt(duration))
    L.append("CFL %s" % _fmt(CFL))
    L.append("pp_max_iter %d" % pp_max_iter)
    L.append("pp_residual %s" % repr(pp_residual))
    L.append("lamb_max_iter %d" % lamb_max_iter)
    L.append("lamb_residual %s" % repr(lamb_residual))
    L.append("lamb_relax %s" % _fmt(lamb_relax))
    L.append("lamb_cut %s" % repr(lamb_cut))
    L.append("")
    L.append("BOUNDARY CONDITIONS")
    L.append("vel_tDelay 0.")
    faces = ["W", "E", "S", "N", "B", "T"]
    L.append("PRESSURE")
    for f in faces:
        ax = faces.index(f) // 2
        L.append("bc.p%s %s" % (f, "PERIODIC" if periodic[ax] else "NEUMANN 0"))
    for comp, title in zip("uvw", ("X-VELOCITY", "Y-VELOCITY", "Z-VELOCITY")):
        L.append(title)
        for f in faces:
            ax = faces.index(f) // 2
            L.append("bc.%s%s %s" % (comp, f, "PERIODIC" if periodic[ax]
                                     else "DIRICHLET 0 0"))
    L.append("")
    L.append("INITIAL CONDITION")
    L.append("init_cond %s" % init_cond)
    L.append("")
    L.append("SOLVABILITY ENFORCEMENT PLANE")
    L.append("out_plane %s" % out_plane)
    L.append("")
    L.append("SIMULATION DRIVING CONDITIONS")
    L.append("p_tDelay 0.")
    for c, v in zip("xyz", gradP):
        L.append("gradP.%s %s 0." % (c, _fmt(v)))
    L.append("g_tDelay 0.")
    for c, v in zip("xyz", g):
        L.append("g.%s %s 0." % (c, _fmt(v)))
    L.append("")
    L.append("PID CONTROLLER GAINS")
    L.append("Kp 0.")
    L.append("Ki 0.")
    L.append("Kd 0.")
    with open(path, "w") as fh:
        fh.write("\n".join(L) + "\n")


def write_part_config(path, parts, loa=0.0):
    """Write part.config; `parts` is a list of dicts with keys r, x, y, z and
    optional rho, order, rsr, translating, rotating."""
    L = ["n %d" % len(parts), "(l/a) %s" % _fmt(loa)]
    for p in parts:
        L.append("")
        L.append("r %s" % _fmt(p["r"]))
        L.append("(x, y, z) %s %s %s" % (_fmt(p["x"]), _fmt(p["y"]), _fmt(p["z"])))
        L.append("(aFx, aFy, aFz) 0. 0. 0.")
        L.append("(aLx, aLy, aLz) 0. 0. 0.")
        L.append("rho %s" % _fmt(p.get("rho", 2.0)))
        L.append("E 1.e6")
        L.append("sigma 0.5")
        L.append("e_dry 1.")
        L.append("coeff_fric 0.5")
        L.append("order %d" % p.get("order", 4))
        L.append("rs/r %s" % _fmt(p.get("rsr", 1.2)))
        L.append("spring_k 0.")
        L.append("spring (x, y, z) 0. 0. 0.")
        L.append("spring_l 0.")
        L.append("translating %d" % p.get("translating", 1))
        L.append("rotating %d" % p.get("rotating", 1))
    with open(path, "w") as fh:
        fh.write("\n".join(L) + "\n")


@dataclass
class Workload:
    """A benchmark/parity configuration: flow.config keys, the seeded pack
    (n spheres of radius a, min surface gap in radii, density, seed) and the
    build-side options."""
    name: str
    flow: dict
    npart: int = 0
    a: float = 1.0
    gap: float = 0.1
    rho_p: float = 2.0
    order: int = 4
    rsr: float = 1.2
    seed: int = 1
    taylor_green: float = 0.0
    loa: float = 0.0
    options: dict = field(default_factory=dict)

    def write(self, dirpath):
        os.makedirs(dirpath, exist_ok=True)
        write_flow_config(os.path.join(dirpath, "flow.config"), **self.flow)
        write_part_config(os.path.join(dirpath, "part.config"), [], loa=self.loa)
        return dirpath


def _box(nx, ny, nz, L):
    return dict(n=(nx, ny, nz), lo=(0.0, 0.0, 0.0), hi=L)


TWO_PI = 6.283185307179586


def taylor_green(n=32, steps_dt=0.01, tol=1e-10):
    """Triply periodic Taylor-Green vortex, L = 2 pi, nu = 0.01, fixed dt."""
    f = _box(n, n, n, (TWO_PI, TWO_PI, TWO_PI))
    f.update(nu=0.01, pp_residual=tol, pp_max_iter=5000, lamb_max_iter=1,
             CFL=0.5)
    return Workload("taylor_green_%d" % n, f, taylor_green=1.0,
                    options=dict(fixed_dt=steps_dt, implicit=1))


def sedimentation(n=(64, 64, 64), side=(16.0, 16.0, 16.0), npart=8, nu=0.1,
                  tol=1e-8, lamb_max_iter=25, dt=None, seed=1, prec=0,
                  gap=0.1, loa=0.0):
    """Periodic box of seeded spheres (radius 1, density ratio 2) settling
    under gravity 1 along -z; the box's net weight is balanced by gradP.z.

    The time step follows the reference's rule (cuda_find_dt,
    src/cuda_bluebottle.cu:3500-3577, Crank-Nicolson form): CFL 0.5 over the
    advective terms, growing at most 1.1x per step from the viscous start
    value of domain_init.  `dt` fixes it instead.  `gap` is the pack's
    minimum surface gap in radii; `loa` the lubrication range l/a of
    part.config (the reference's collision_parts acts for gaps below
    int(l/a) radii, src/bluebottle_kernel.cu:2597)."""
    f = _box(n[0], n[1], n[2], side)
    f.update(nu=nu, pp_residual=tol, pp_max_iter=20000, CFL=0.5,
             lamb_max_iter=lamb_max_iter, lamb_residual=1e-2, g=(0.0, 0.0, -1.0),
             lamb_cut=1e-4, lamb_relax=1.0)
    opts = dict(implicit=1, gravity_balance=1, precision=prec)
    if dt is not None:
        opts["fixed_dt"] = dt
    return Workload("sediment_%dx%dx%d_%dp" % (n[0], n[1], n[2], npart), f,
                    npart=npart, seed=seed, gap=gap, loa=loa, options=opts)


# The benchmark configurations C1-C5: Taylor-Green 32^3, then sedimenting
# sphere packs from 64^3 + 8 spheres to 256x256x512 + 8000 spheres (seeded
# synthetic inputs of those shapes).  The 8-sphere pack keeps its 0.1-radius
# minimum gap; the dense packs are seeded 0.5 radii apart (2 cells at 4
# cells per radius) and carry the reference's default lubrication range
# l/a = 1 (sim/input/part.config).  At 4 cells per radius a pair closer than
# about 0.12 radii has quadrature nodes (rs = 1.2 a) inside its partner,
# which the reference's check_nodes screens for walls only
# (src/quadrature_kernel.cu:45-96), and the flow in that gap diverges
# within a few steps, in either precision form.
DENSE_GAP = 0.5
DENSE_LOA = 1.0


def config_c1():
    return taylor_green(32)


def config_c2():
    return sedimentation((64, 64, 64), (16.0, 16.0, 16.0), 8, nu=0.1)


def config_c3(prec=1):
    return sedimentation((128, 128, 128), (32.0, 32.0, 32.0), 256, nu=0.1,
                         prec=prec, gap=DENSE_GAP, loa=DENSE_LOA)


def config_c4(prec=0):
    return sedimentation((256, 256, 256), (64.0, 64.0, 64.0), 2000, nu=0.05,
                         prec=prec, gap=DENSE_GAP, loa=DENSE_LOA)


def config_c5(prec=1, lamb_max_iter=25):
    return sedimentation((256, 256, 512), (64.0, 64.0, 128.0), 8000, nu=0.05,
                         prec=prec, lamb_max_iter=lamb_max_iter, gap=DENSE_GAP,
                         loa=DENSE_LOA)
