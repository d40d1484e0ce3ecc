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

/* The values one face of component C (0 = u on Gfx, 1 = v on Gfy, 2 = w
 * on Gfz) reads: its own velocity x0 and its neighbours m[a] / pl[a] one
 * step down / up along axis a; for each transverse axis a != C the four
 * a-velocities t[a][0..3] at the faces bracketing this one (t0 = at
 * -OFF(a, C), t1 = at the same index, t2 = at -OFF(a, C) + OFF(a, a), t3 =
 * at +OFF(a, a), on grid a); the pressures pa = p0 one cell down along C
 * and pb = p0 at the face's cell; conv0 (and, explicit form, diff0 and
 * whether both cells are fluid). */
struct rhs_in {
  double x0, m[3], pl[3], t[3][4];
  double pa, pb, conv0, diff0;
  int fluid;
};

/* the right-hand side of one face from its gathered values: arithmetic,
 * including the order of every sum, of ustar_rhs / vstar_rhs / wstar_rhs
 * (src/bicgstab_kernel.cu:27-481) and u_star_2 / v_star_2 / w_star_2
 * (src/bluebottle_kernel.cu:1504-2004) */
template <int C>
__device__ __forceinline__ void rhs_eval(const rhs_args &A, const rhs_in &I,
  double &s_out, double &cv_out, double &df_out)
{
  const bbb_geom &G = A.G;
  const double dd[3] = {1. / G.dx, 1. / G.dy, 1. / G.dz};
  const double x0 = I.x0;
  double s = (I.pa - I.pb) * dd[C] / A.rho_f;
  double term[3];
#pragma unroll
  for(int a = 0; a < 3; a++) {
    double t;
    if(a == C) {
      t = (I.pl[a] + x0) * (I.pl[a] + x0) - (x0 + I.m[a]) * (x0 + I.m[a]);
    } else {
      t = (I.pl[a] + x0) * (I.t[a][3] + I.t[a][2])
        - (x0 + I.m[a]) * (I.t[a][1] + I.t[a][0]);
    }
    term[a] = t * (0.25 * dd[a]);
  }
  double cv = term[0] + term[1] + term[2];
  if(A.dt0 > 0) s += (-A.ab * cv + A.ab0 * I.conv0);
  else s += -cv;
  double lap[3];
#pragma unroll
  for(int a = 0; a < 3; a++) {
    double d1 = (I.pl[a] - x0) * dd[a];
    double d0 = (x0 - I.m[a]) * dd[a];
    lap[a] = (d1 - d0) * dd[a];
  }
  double df = A.nu * (lap[0] + lap[1] + lap[2]);
  if(A.explicit_ab2) {
    if(A.dt0 > 0) s += (A.ab * df - A.ab0 * I.diff0);
    else s += df;
  } else {
    s += 0.5 * df;
  }
  s += A.f[C];
  s *= A.dt;
  s += x0;
  if(A.explicit_ab2) s *= I.fluid;
  s_out = s;
  cv_out = cv;
  df_out = df;
}

/* one face of component C at (i, j, k), its values read through L1 */
template <int C>
__device__ __forceinline__ void rhs_component(const rhs_args &A, int i, int j,
  int k)
{
  const bbb_geom &G = A.G;
  const int s1[3] = {G.fx_s1, G.fy_s1, G.fz_s1};
  const int s2[3] = {G.fx_s2, G.fy_s2, G.fz_s2};
  const real *vel[3] = {A.u0, A.v0, A.w0};
  /* offsets of a unit step along x, y, z in grid g */
#define OFF(g, a) ((a) == 0 ? 1LL : ((a) == 1 ? (long long)s1[g] : (long long)s2[g]))
  long long Cc = i + (long long)j * s1[C] + (long long)k * s2[C];
  long long Cp = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
  long long cstep = C == 0 ? 1LL : (C == 1 ? (long long)G.cc_s1 : (long long)G.cc_s2);
  const real *vc = vel[C];
  rhs_in I;
  I.x0 = __ldg(vc + Cc);
#pragma unroll
  for(int a = 0; a < 3; a++) {
    I.m[a] = __ldg(vc + Cc - OFF(C, a));
    I.pl[a] = __ldg(vc + Cc + OFF(C, a));
    if(a != C) {
      const real *vt = vel[a];
      long long Ct = i + (long long)j * s1[a] + (long long)k * s2[a];
      I.t[a][0] = __ldg(vt + Ct - OFF(a, C));
      I.t[a][1] = __ldg(vt + Ct);
      I.t[a][2] = __ldg(vt + Ct - OFF(a, C) + OFF(a, a));
      I.t[a][3] = __ldg(vt + Ct + OFF(a, a));
    }
  }
  I.pa = __ldg(A.p0 + Cp - cstep);
  I.pb = __ldg(A.p0 + Cp);
  I.conv0 = A.dt0 > 0 ? __ldg(A.conv0[C] + Cc) : 0.;
  I.diff0 = 0.;
  I.fluid = 1;
  if(A.explicit_ab2) {
    I.diff0 = A.dt0 > 0 ? __ldg(A.diff0[C] + Cc) : 0.;
    I.fluid = __ldg(A.phase + Cp - cstep) < 0 && __ldg(A.phase + Cp) < 0;
  }
  double s, cv, df;
  rhs_eval<C>(A, I, s, cv, df);
  if(A.explicit_ab2) A.diff[C][Cc] = df;
  A.star[C][Cc] = s;
  A.conv[C][Cc] = cv;
#undef OFF
}

/* All three components in one pass (the explicit form): a block owns a
 * 32 x 8 tile of (i, j) of the union of the three face index spaces and
 * marches through RHS_KZ planes along k. */
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

/* One component of the Crank-Nicolson form (the Helmholtz solves' right-
 * hand sides, one component per call).  A warp owns 32 consecutive faces
 * of one row (i) and a block 8 rows (j); the block marches RHS_KZC planes
 * along k.  Values along z stay in registers from one plane to the next
 * (the component's own k - 1, k, k + 1 and the transverse velocities and
 * pressures a face reads at two planes), values at i - 1 / i + 1 come from
 * the neighbouring lanes by shuffles (lanes 0 and 31 read their outer
 * neighbour themselves), the rest are plain coalesced loads: 8 loads per
 * face of u and w, 10 of v, instead of 18.  The arithmetic is rhs_eval's,
 * as in rhs_component (the compiler may fuse a multiply-add differently in
 * the two kernels: a last-bit difference at most). */
#define RHS_KZC 16
/* resident blocks per SM the register budget targets: 3 (80 registers, a
 * few values spilled) measured 0.495 ms per component at 256x256x512
 * against 0.598 ms at 2 blocks with every value in registers and 0.576 ms
 * for rhs_component one face per thread */
#ifndef BBB_RHS_MINB
#define BBB_RHS_MINB 3
#endif

template <int C>
__global__ void __launch_bounds__(256, BBB_RHS_MINB) k_star_rhs_z(rhs_args A)
{
  const bbb_geom &G = A.G;
  const int lane = threadIdx.x;                 /* blockDim.x == 32 */
  const int i = blockIdx.x * 32 + lane + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  /* the face index space of component C */
  const int imax = C == 0 ? G.nx + 1 : G.nx;
  const int jmax = C == 1 ? G.ny + 1 : G.ny;
  const int kmax = C == 2 ? G.nz + 1 : G.nz;
  if(j > jmax) return;                          /* whole warp: one row */
  const bool act = i <= imax;
  const int k0 = blockIdx.z * RHS_KZC + 1;
  const int k1 = min(k0 + RHS_KZC, kmax + 1);
  if(k0 >= k1) return;                          /* whole block */
  const unsigned FULL = 0xffffffffu;
  /* x index each lane loads (its own face, held inside every array's
   * ghosted x extent), and the outer neighbours lanes 0 and 31 load */
  const int ifx = min(i, G.fx_s1 - 1), icc = min(i, G.cc_s1 - 1);
  const int ilo = i - 1;                        /* >= 0 */
  const int ihx = min(i + 1, G.fx_s1 - 1), ihc = min(i + 1, G.cc_s1 - 1);
  const real *U = A.u0, *V = A.v0, *W = A.w0, *P = A.p0;
  auto fx = [&](int ii, int jj, int kk) { return ii + (long long)jj * G.fx_s1 + (long long)kk * G.fx_s2; };
  auto fy = [&](int ii, int jj, int kk) { return ii + (long long)jj * G.fy_s1 + (long long)kk * G.fy_s2; };
  auto fz = [&](int ii, int jj, int kk) { return ii + (long long)jj * G.fz_s1 + (long long)kk * G.fz_s2; };
  auto cc = [&](int ii, int jj, int kk) { return ii + (long long)jj * G.cc_s1 + (long long)kk * G.cc_s2; };
  /* value at i - 1 / i + 1 of a lane-distributed row value */
  auto west = [&](double v, double edge) {
    double r = __shfl_up_sync(FULL, v, 1);
    return lane == 0 ? edge : r;
  };
  auto east = [&](double v, double edge) {
    double r = __shfl_down_sync(FULL, v, 1);
    return lane == 31 ? edge : r;
  };
  if constexpr(C == 0) {
    /* u at (i, j, k); v at (i - 1 | i, j | j + 1, k); w at (i - 1 | i,
     * j, k | k + 1); p at (i - 1 | i, j, k) */
    double um = __ldg(U + fx(ifx, j, k0 - 1)), uc = __ldg(U + fx(ifx, j, k0));
    double wc = __ldg(W + fz(icc, j, k0));
    double wcw = lane == 0 ? __ldg(W + fz(ilo, j, k0)) : 0.;
    wcw = west(wc, wcw);
#pragma unroll 1
    for(int k = k0; k < k1; k++) {
      const double un = __ldg(U + fx(ifx, j, k + 1));
      const double us = __ldg(U + fx(ifx, j - 1, k)), uN = __ldg(U + fx(ifx, j + 1, k));
      const double v0 = __ldg(V + fy(icc, j, k)), v1 = __ldg(V + fy(icc, j + 1, k));
      const double wn = __ldg(W + fz(icc, j, k + 1));
      const double pc = __ldg(P + cc(icc, j, k));
      double e_uw = 0., e_ue = 0., e_v0 = 0., e_v1 = 0., e_wn = 0., e_p = 0.;
      if(lane == 0) {
        e_uw = __ldg(U + fx(ilo, j, k)); e_v0 = __ldg(V + fy(ilo, j, k));
        e_v1 = __ldg(V + fy(ilo, j + 1, k)); e_wn = __ldg(W + fz(ilo, j, k + 1));
        e_p = __ldg(P + cc(ilo, j, k));
      }
      if(lane == 31) e_ue = __ldg(U + fx(ihx, j, k));
      rhs_in I;
      I.x0 = uc;
      I.m[0] = west(uc, e_uw); I.pl[0] = east(uc, e_ue);
      I.m[1] = us; I.pl[1] = uN;
      I.m[2] = um; I.pl[2] = un;
      I.t[1][0] = west(v0, e_v0); I.t[1][1] = v0;
      I.t[1][2] = west(v1, e_v1); I.t[1][3] = v1;
      const double wnw = west(wn, e_wn);
      I.t[2][0] = wcw; I.t[2][1] = wc; I.t[2][2] = wnw; I.t[2][3] = wn;
      I.pa = west(pc, e_p); I.pb = pc;
      const long long Cc = fx(i, j, k);
      I.conv0 = (act && A.dt0 > 0) ? __ldg(A.conv0[0] + Cc) : 0.;
      I.diff0 = 0.; I.fluid = 1;
      if(act) {
        double sv, cv, df;
        rhs_eval<0>(A, I, sv, cv, df);
        A.star[0][Cc] = sv;
        A.conv[0][Cc] = cv;
      }
      um = uc; uc = un; wc = wn; wcw = wnw;
    }
  } else if constexpr(C == 1) {
    /* v at (i, j, k); u at (i | i + 1, j - 1 | j, k); w at (i, j - 1 | j,
     * k | k + 1); p at (i, j - 1 | j, k) */
    double vm = __ldg(V + fy(icc, j, k0 - 1)), vc = __ldg(V + fy(icc, j, k0));
    double ws = __ldg(W + fz(icc, j - 1, k0)), wc = __ldg(W + fz(icc, j, k0));
#pragma unroll 1
    for(int k = k0; k < k1; k++) {
      const double vn = __ldg(V + fy(icc, j, k + 1));
      const double vS = __ldg(V + fy(icc, j - 1, k)), vN = __ldg(V + fy(icc, j + 1, k));
      const double u0 = __ldg(U + fx(ifx, j - 1, k)), u1 = __ldg(U + fx(ifx, j, k));
      const double wsn = __ldg(W + fz(icc, j - 1, k + 1)), wcn = __ldg(W + fz(icc, j, k + 1));
      const double ps = __ldg(P + cc(icc, j - 1, k)), pc = __ldg(P + cc(icc, j, k));
      double e_vw = 0., e_ve = 0., e_u0 = 0., e_u1 = 0.;
      if(lane == 0) e_vw = __ldg(V + fy(ilo, j, k));
      if(lane == 31) {
        e_ve = __ldg(V + fy(ihc, j, k));
        e_u0 = __ldg(U + fx(ihx, j - 1, k)); e_u1 = __ldg(U + fx(ihx, j, k));
      }
      rhs_in I;
      I.x0 = vc;
      I.m[0] = west(vc, e_vw); I.pl[0] = east(vc, e_ve);
      I.m[1] = vS; I.pl[1] = vN;
      I.m[2] = vm; I.pl[2] = vn;
      I.t[0][0] = u0; I.t[0][1] = u1;
      I.t[0][2] = east(u0, e_u0); I.t[0][3] = east(u1, e_u1);
      I.t[2][0] = ws; I.t[2][1] = wc; I.t[2][2] = wsn; I.t[2][3] = wcn;
      I.pa = ps; I.pb = pc;
      const long long Cc = fy(i, j, k);
      I.conv0 = (act && A.dt0 > 0) ? __ldg(A.conv0[1] + Cc) : 0.;
      I.diff0 = 0.; I.fluid = 1;
      if(act) {
        double sv, cv, df;
        rhs_eval<1>(A, I, sv, cv, df);
        A.star[1][Cc] = sv;
        A.conv[1][Cc] = cv;
      }
      vm = vc; vc = vn; ws = wsn; wc = wcn;
    }
  } else {
    /* w at (i, j, k); u at (i | i + 1, j, k - 1 | k); v at (i, j | j + 1,
     * k - 1 | k); p at (i, j, k - 1 | k) */
    double wm = __ldg(W + fz(icc, j, k0 - 1)), wc = __ldg(W + fz(icc, j, k0));
    double um = __ldg(U + fx(ifx, j, k0 - 1));
    double ume = lane == 31 ? __ldg(U + fx(ihx, j, k0 - 1)) : 0.;
    ume = east(um, ume);
    double v0m = __ldg(V + fy(icc, j, k0 - 1)), v1m = __ldg(V + fy(icc, j + 1, k0 - 1));
    double pm = __ldg(P + cc(icc, j, k0 - 1));
#pragma unroll 1
    for(int k = k0; k < k1; k++) {
      const double wn = __ldg(W + fz(icc, j, k + 1));
      const double wS = __ldg(W + fz(icc, j - 1, k)), wN = __ldg(W + fz(icc, j + 1, k));
      const double uk = __ldg(U + fx(ifx, j, k));
      const double v0 = __ldg(V + fy(icc, j, k)), v1 = __ldg(V + fy(icc, j + 1, k));
      const double pc = __ldg(P + cc(icc, j, k));
      double e_ww = 0., e_we = 0., e_uk = 0.;
      if(lane == 0) e_ww = __ldg(W + fz(ilo, j, k));
      if(lane == 31) { e_we = __ldg(W + fz(ihc, j, k)); e_uk = __ldg(U + fx(ihx, j, k)); }
      rhs_in I;
      I.x0 = wc;
      I.m[0] = west(wc, e_ww); I.pl[0] = east(wc, e_we);
      I.m[1] = wS; I.pl[1] = wN;
      I.m[2] = wm; I.pl[2] = wn;
      const double uke = east(uk, e_uk);
      I.t[0][0] = um; I.t[0][1] = uk; I.t[0][2] = ume; I.t[0][3] = uke;
      I.t[1][0] = v0m; I.t[1][1] = v0; I.t[1][2] = v1m; I.t[1][3] = v1;
      I.pa = pm; I.pb = pc;
      const long long Cc = fz(i, j, k);
      I.conv0 = (act && A.dt0 > 0) ? __ldg(A.conv0[2] + Cc) : 0.;
      I.diff0 = 0.; I.fluid = 1;
      if(act) {
        double sv, cv, df;
        rhs_eval<2>(A, I, sv, cv, df);
        A.star[2][Cc] = sv;
        A.conv[2][Cc] = cv;
      }
      wm = wc; wc = wn; um = uk; ume = uke; v0m = v0; v1m = v1; pm = pc;
    }
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
  if(!explicit_ab2 && (comp_mask == 1 || comp_mask == 2 || comp_mask == 4)) {
    const int C = comp_mask == 1 ? 0 : (comp_mask == 2 ? 1 : 2);
    const int ni = C == 0 ? A.G.nx + 1 : A.G.nx;
    const int nj = C == 1 ? A.G.ny + 1 : A.G.ny;
    const int nk = C == 2 ? A.G.nz + 1 : A.G.nz;
    dim3 g1((ni + 31) / 32, (nj + 7) / 8, (nk + RHS_KZC - 1) / RHS_KZC);
    if(C == 0) k_star_rhs_z<0><<<g1, blk, 0, g_dev.stream>>>(A);
    else if(C == 1) k_star_rhs_z<1><<<g1, blk, 0, g_dev.stream>>>(A);
    else k_star_rhs_z<2><<<g1, blk, 0, g_dev.stream>>>(A);
  } else {
    k_star_rhs<<<grd, blk, 0, g_dev.stream>>>(A);
  }
  BBB_LAUNCHED();
  bbb_prof_end();
}

/* src/cuda_bluebottle.cu:2930-3026 */
extern "C" void cuda_U_star_2(void) { bbb_star_rhs(7, 1); }

/* src/cuda_bicgstab.cu:1091-1175 */
extern "C" void cuda_ustar_rhs(int dev) { (void)dev; bbb_star_rhs(1, 0); }
extern "C" void cuda_vstar_rhs(int dev) { (void)dev; bbb_star_rhs(2, 0); }
extern "C" void cuda_wstar_rhs(int dev) { (void)dev; bbb_star_rhs(4, 0); }
