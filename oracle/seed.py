"""Seeded sphere pack and benchmark input files, restated for the CPU side.

TEST INFRASTRUCTURE ONLY: used by tests/ and by bench.py's CPU legs to set
up a workload without the product library.  It restates the library's
seeded packer (bbb_seed_particles), which follows the placement rules of the
reference's seeder (src/seeder.c:220-300: centres inside the domain less
its screens, at least a radius from a non-periodic wall, periodic images
only along periodic axes) with a reproducible splitmix64 stream in place of
srand(time(NULL)) (src/seeder.c:234) and a minimum surface gap.  The pack is
bit-identical to the library's (tests/test_host.py checks it), so the
reference's own readers (oracle/_ref/libref_host*.so) can load the same
particles from part.config.
"""
import math
import os

M64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
    generators", OOPSLA 2014) and doubles in [0, 1) from its top 53 bits."""

    def __init__(self, seed):
        self.s = seed & M64

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & M64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)

    def uniform(self):
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)


def c_round(x):
    """C's round(): halves away from zero (Python's round() is to even)."""
    t = math.trunc(x)
    if abs(x - t) >= 0.5:
        t += 1 if x > 0 else -1
    return float(t)


class _Axis:
    def __init__(self, xs, xl, ds_lo, ds_hi, per, wall, dmin):
        self.origin, self.L, self.per = xs, xl, per
        self.lo = xs + ds_lo + (0.0 if per else wall)
        self.len = xl - ds_lo - ds_hi - (0.0 if per else 2.0 * wall)
        self.nc = max(1, int(math.floor(xl / dmin)))

    def cell(self, x):
        c = int((x - self.origin) / self.L * self.nc)
        return min(max(c, 0), self.nc - 1)


def seed_pack(n, lo, hi, periodic, a=1.0, min_gap=0.1, seed=1,
              screens=(0.0,) * 6):
    """Centres of n spheres of radius a, surface gap >= min_gap*a (periodic
    images along the periodic axes), as a list of (x, y, z); None when the
    pack cannot be placed within the library's try budget."""
    dmin = 2.0 * a + min_gap * a
    wall = a + 0.5 * min_gap * a
    axes = [_Axis(lo[d], hi[d] - lo[d], screens[2 * d], screens[2 * d + 1],
                  periodic[d], wall, dmin) for d in range(3)]
    if any(ax.len <= 0 for ax in axes) and n > 0:
        return None
    rng = SplitMix64(seed)
    head = {}
    pts = []
    tries, max_tries = 0, 2000 * max(n, 1) + 100000
    while len(pts) < n and tries < max_tries:
        tries += 1
        p = [0.0, 0.0, 0.0]
        ic = [0, 0, 0]
        for d in range(3):
            p[d] = axes[d].lo + rng.uniform() * axes[d].len
            ic[d] = axes[d].cell(p[d])
        ok = True
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    off = (dx, dy, dz)
                    jc = [0, 0, 0]
                    inside = True
                    for d in range(3):
                        jc[d] = ic[d] + off[d]
                        if axes[d].per:
                            jc[d] %= axes[d].nc
                        elif jc[d] < 0 or jc[d] >= axes[d].nc:
                            inside = False
                    for d in range(3):
                        if inside and axes[d].per and axes[d].nc < 3 and off[d] != 0 \
                                and (axes[d].nc == 1 or off[d] == 1):
                            inside = False
                    if not inside:
                        continue
                    for q in head.get(tuple(jc), ()):
                        r2 = 0.0
                        for d in range(3):
                            r = p[d] - pts[q][d]
                            if axes[d].per:
                                r -= axes[d].L * c_round(r / axes[d].L)
                            r2 += r * r
                        if r2 < dmin * dmin:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        head.setdefault(tuple(ic), []).append(len(pts))
        pts.append(tuple(p))
    return pts if len(pts) == n else None


def gravity_balance(n, a, rho_p, rho_f, g_z, box_volume):
    """gradP.z that makes the periodic box's net weight zero, summed in the
    library's order (bbb_parts_init, option gravity_balance)."""
    ex = 0.0
    for _ in range(n):
        ex += (rho_p - rho_f) * 4. / 3. * math.pi * a * a * a
    return ex * g_z / box_volume


def write_workload_inputs(wl, dirpath):
    """flow.config and part.config of a configs.Workload with its seeded pack
    written out and the gravity balance folded into gradP.z, so that the
    reference's own readers set up the same state the library does.
    Returns the input directory."""
    from bluebottle_b200 import configs
    os.makedirs(dirpath, exist_ok=True)
    flow = dict(wl.flow)
    lo = flow.get("lo", (0.0, 0.0, 0.0))
    hi = flow["hi"]
    periodic = flow.get("periodic", (True, True, True))
    parts = []
    if wl.npart > 0:
        pts = seed_pack(wl.npart, lo, hi, periodic, wl.a, wl.gap, wl.seed)
        if pts is None:
            raise RuntimeError("particle pack too dense for the box")
        parts = [dict(r=wl.a, x=x, y=y, z=z, rho=wl.rho_p, order=wl.order,
                      rsr=wl.rsr) for (x, y, z) in pts]
    if wl.options.get("gravity_balance"):
        vol = (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2])
        gz = flow.get("g", (0.0, 0.0, 0.0))[2]
        gp = list(flow.get("gradP", (0.0, 0.0, 0.0)))
        gp[2] = gravity_balance(wl.npart, wl.a, wl.rho_p, flow.get("rho_f", 1.0),
                                gz, vol)
        flow["gradP"] = tuple(gp)
    configs.write_flow_config(os.path.join(dirpath, "flow.config"), **flow)
    # repr() of a double reads back to the same double through %lf
    configs.write_part_config(os.path.join(dirpath, "part.config"), parts,
                              loa=wl.loa)
    return dirpath
