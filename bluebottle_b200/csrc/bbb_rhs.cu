/* bbb_rhs.cu -- momentum right-hand sides on the staggered grid.
 *
 * One kernel computes u*, v* and w* together: a thread owns index (i,j,k)
 * of the union of the three face index spaces and evaluates every
 * component whose face exists there.  All three velocity components are
 * read once per tile through L1, so the fused pass reads u0, v0, w0, p0 and
 * the three conv0 fields and writes u*, v*, w* and the three conv fields:
 * 13 words per cell (Crank-Nicolson form).
 *
 * Arithmetic, including the order of every sum, follows
 * ustar_rhs / vstar_rhs / wstar_rhs (src/bicgstab_kernel.cu:27-481) for the
 * Crank-Nicolson form and u_star_2 / v_star_2 / w_star_2
 * (src/bluebottle_kernel.cu:1504-2004) for the explicit Adams-Bashforth
 * form.  The uniform forcing -gradP/rho_f enters as a scalar.
 */
#include "bbb_internal.h"

struct rhs_args {
  const real *u0, *v0, *w0, *p0;
  const real *conv0[3], *diff0[3];
  real *star[3], *conv[3], *diff[3];
  const int *phase;
  bbb_geom G;
  double rho_f, nu, dt, dt0, ab, ab0;
  double f[3];
  int comp_mask;
  int explicit_ab2;
};

/* component along axis C (0 = u on Gfx, 1 = v on Gfy, 2 = w on Gfz) */
template <int C>
__device__ __forceinline__ void rhs_component(const rhs_args &A, int i, int j,
  int k)
{
  const bbb_geom &G = A.G;
  const int s1[3] = {G.fx_s1, G.fy_s1, G.fz_s1};
  const int s2[3] = {G.fx_s2, G.fy_s2, G.fz_s2};
  const real *vel[3] = {A.u0, A.v0, A.w0};
  const double dd[3] = {1. / G.dx, 1. / G.dy, 1. / G.dz};
  /* offsets of a unit step along x, y, z in grid g */
#define OFF(g, a) ((a) == 0 ? 1LL : ((a) == 1 ? (long long)s1[g] : (long long)s2[g]))
  long long Cc = i + (long long)j * s1[C] + (long long)k * s2[C];
  long long Cp = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
  long long cstep = C == 0 ? 1LL : (C == 1 ? (long long)G.cc_s1 : (long long)G.cc_s2);
  const real *vc = vel[C];
  double x0 = __ldg(vc + Cc);
  double m[3], pl[3];
#pragma unroll
  for(int a = 0; a < 3; a++) {
    m[a] = __ldg(vc + Cc - OFF(C, a));
    pl[a] = __ldg(vc + Cc + OFF(C, a));
  }
  double s = (__ldg(A.p0 + Cp - cstep) - __ldg(A.p0 + Cp)) * dd[C] / A.rho_f;
  double term[3];
#pragma unroll
  for(int a = 0; a < 3; a++) {
    double t;
    if(a == C) {
      t = (pl[a] + x0) * (pl[a] + x0) - (x0 + m[a]) * (x0 + m[a]);
    } else {
      /* transverse component along a at the faces bracketing this one */
      const real *vt = vel[a];
      long long Ct = i + (long long)j * s1[a] + (long long)k * s2[a];
      double t0 = __ldg(vt + Ct - OFF(a, C));
      double t1 = __ldg(vt + Ct);
      double t2 = __ldg(vt + Ct - OFF(a, C) + OFF(a, a));
      double t3 = __ldg(vt + Ct + OFF(a, a));
      t = (pl[a] + x0) * (t3 + t2) - (x0 + m[a]) * (t1 + t0);
    }
    term[a] = t * (0.25 * dd[a]);
  }
  double cv = term[0] + term[1] + term[2];
  if(A.dt0 > 0) s += (-A.ab * cv + A.ab0 * __ldg(A.conv0[C] + Cc));
  else s += -cv;
  double lap[3];
#pragma unroll
  for(int a = 0; a < 3; a++) {
    double d1 = (pl[a] - x0) * dd[a];
    double d0 = (x0 - m[a]) * dd[a];
    lap[a] = (d1 - d0) * dd[a];
  }
  double df = A.nu * (lap[0] + lap[1] + lap[2]);
  if(A.explicit_ab2) {
    if(A.dt0 > 0) s += (A.ab * df - A.ab0 * __ldg(A.diff0[C] + Cc));
    else s += df;
  } else {
    s += 0.5 * df;
  }
  s += A.f[C];
  s *= A.dt;
  s += x0;
  if(A.explicit_ab2) {
    s *= (__ldg(A.phase + Cp - cstep) < 0 && __ldg(A.phase + Cp) < 0);
    A.diff[C][Cc] = df;
  }
  A.star[C][Cc] = s;
  A.conv[C][Cc] = cv;
#undef OFF
}

/* A block owns a 32 x 8 tile of (i, j) and marches through RHS_KZ planes
 * along k, so the k - 1 and k + 1 neighbours a thread reads were read by
 * the same block one plane earlier and come from L1, not L2. */
#define RHS_KZ 8

__global__ void __launch_bounds__(256) k_star_rhs(rhs_args A)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const bbb_geom &G = A.G;
  if(i > G.nx + 1 || j > G.ny + 1) return;
  const int k0 = blockIdx.z * RHS_KZ + 1;
  const int k1 = min(k0 + RHS_KZ, G.nz + 2);
#pragma unroll 1
  for(int k = k0; k < k1; k++) {
    if((A.comp_mask & 1) && j <= G.ny && k <= G.nz) rhs_component<0>(A, i, j, k);
    if((A.comp_mask & 2) && i <= G.nx && k <= G.nz) rhs_component<1>(A, i, j, k);
    if((A.comp_mask & 4) && i <= G.nx && j <= G.ny) rhs_component<2>(A, i, j, k);
  }
}

void bbb_star_rhs(int comp_mask, int explicit_ab2)
{
  bbb_dev_require();
  if(!g_dev.ready) return;
  rhs_args A;
  A.u0 = g_dev.u0; A.v0 = g_dev.v0; A.w0 = g_dev.w0; A.p0 = g_dev.p0;
  A.conv0[0] = g_dev.conv0_u; A.conv0[1] = g_dev.conv0_v; A.conv0[2] = g_dev.conv0_w;
  A.diff0[0] = g_dev.diff0_u; A.diff0[1] = g_dev.diff0_v; A.diff0[2] = g_dev.diff0_w;
  A.star[0] = g_dev.us; A.star[1] = g_dev.vs; A.star[2] = g_dev.ws;
  A.conv[0] = g_dev.conv_u; A.conv[1] = g_dev.conv_v; A.conv[2] = g_dev.conv_w;
  A.diff[0] = g_dev.diff_u; A.diff[1] = g_dev.diff_v; A.diff[2] = g_dev.diff_w;
  A.phase = g_dev.phase;
  A.G = bbb_make_geom();
  A.rho_f = rho_f; A.nu = nu; A.dt = dt; A.dt0 = dt0;
  A.ab0 = 0.5 * dt / dt0;
  A.ab = 1. + A.ab0;
  A.f[0] = -gradP.x / rho_f; A.f[1] = -gradP.y / rho_f; A.f[2] = -gradP.z / rho_f;
  A.comp_mask = comp_mask;
  A.explicit_ab2 = explicit_ab2;
  dim3 blk(32, 8), grd((A.G.nx + 1 + 31) / 32, (A.G.ny + 1 + 7) / 8,
    (A.G.nz + 1 + RHS_KZ - 1) / RHS_KZ);
  /* algorithmic words per cell: u0, v0, w0 and p0, read by every
   * component, once; per component conv0 read, star and conv written
   * (+ diff0 read and diff written in the explicit form) */
  int ncomp = (comp_mask & 1) + ((comp_mask >> 1) & 1) + ((comp_mask >> 2) & 1);
  double words = ncomp * (explicit_ab2 ? 5. : 3.) + 4.;
  bbb_prof_begin(BBB_PROF_RHS, (double)A.G.nx * A.G.ny * A.G.nz * words * sizeof(real));
  k_star_rhs<<<grd, blk, 0, g_dev.stream>>>(A);
  BBB_LAUNCHED();
  bbb_prof_end();
}

/* src/cuda_bluebottle.cu:2930-3026 */
extern "C" void cuda_U_star_2(void) { bbb_star_rhs(7, 1); }

/* src/cuda_bicgstab.cu:1091-1175 */
extern "C" void cuda_ustar_rhs(int dev) { (void)dev; bbb_star_rhs(1, 0); }
extern "C" void cuda_vstar_rhs(int dev) { (void)dev; bbb_star_rhs(2, 0); }
extern "C" void cuda_wstar_rhs(int dev) { (void)dev; bbb_star_rhs(4, 0); }
