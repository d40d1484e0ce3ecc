/* bbb_krylov.cu -- matrix-free Jacobi-preconditioned Krylov solvers.
 *
 * Replaces the reference's CUSP calls (src/cuda_bicgstab.cu:44-1073):
 * the 13-diagonal DIA matrices it rebuilds every call (13 words per row,
 * src/bicgstab_kernel.cu:643-1856) are never formed.  One byte per unknown
 * holds the six face weights |flag| and the identity-row bit; the operator
 * is applied from that byte inside the fused kernels, with the diagonal and
 * the Jacobi scale of the 128 possible bytes tabulated in shared memory.
 *
 * BiCGSTAB is CUSP's right-preconditioned krylov::bicgstab (M = diag^-1):
 *   v = A M p;  alpha = rho / (rh, v);  s = r - alpha v;  t = A M s;
 *   omega = (t, s) / (t, t);  x += alpha M p + omega M s;  r = s - omega t;
 *   rho' = (rh, r);  beta = (rho' / rho)(alpha / omega);
 *   p = r + beta p - beta omega v
 * run as two fused stencil passes per iteration, all scalars on the device:
 *   A  r = s - omega t;  x += alpha M p + omega M s;
 *      p = r + beta p - beta omega v;  v = A M p;
 *      (r, r) (rh, r) (rh, v) sum x          -> alpha, convergence
 *   B  s = r - alpha v;  t = A M s;
 *      (t, s) (t, t) (s, s) (rh, s) (rh, t)  -> omega, beta
 * beta needs rho' before pass A forms r, so pass B supplies it as
 * (rh, s) - omega (rh, t), which equals (rh, r) in exact arithmetic; alpha
 * uses the (rh, r) pass A sums.  15 vector words + 2 mask bytes per unknown
 * and iteration.  Stopping rule of CUSP's monitor: ||r|| <= rtol ||b||,
 * iteration count advanced once per full iteration, early exit (without
 * counting) when ||s|| meets it.
 *
 * CG (CUSP's krylov::cg, used for the Crank-Nicolson Helmholtz solves):
 *   C1  p = M r + beta p;  y = A p;  (y, p)
 *   C2  x += alpha p;  r -= alpha y;  (r, M r) (r, r)
 *
 * Stencil kernels tile x-y with 32x8 threads and march along z; the grid
 * is one wave of resident blocks, each taking an equal run of (tile,
 * plane) units, so no block idles at the end.  Where the row length
 * allows, each thread owns V consecutive cells in x (V = 4 for FP32, 2 for
 * FP64: one 128-bit access per array); x neighbours come from registers and
 * warp shuffles, y neighbours from a three-plane shared-memory ring (one
 * barrier per plane), z neighbours from registers.  Rows of other lengths
 * use a one-cell-per-thread tile.
 */
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <mutex>
#include "bbb_internal.h"
#include "bbb_reduce.cuh"

#define TX 32
#define TY 8
#define HX (TX + 2)
#define HY (TY + 2)
#define NTHR (TX * TY)
#define NPW 1184          /* blocks of the pointwise passes (8 per SM) */
#ifndef BBB_KRY_MINB
#define BBB_KRY_MINB 4    /* resident blocks per SM the BiCGSTAB passes target */
#endif

/* operator constants in the form the kernels use */
struct opc {
  double wx, wy, wz;   /* Poisson: +|f|/dx^2; Helmholtz: 0.5 nu dt/dx^2 */
  int helm;
};

/* A box of nx*ny*nz unknowns cut into x-y tiles; the work units are
 * (tile, plane) pairs, tile-major, and block b marches through units
 * [b chunk, (b+1) chunk): one or two z-segments of one or two tiles. */
struct boxc {
  int nx, ny, nz;
  int wW, wE, wS, wN, wB, wT;   /* wrapped neighbour index at each edge */
  int vec;                      /* cells per thread along x            */
  int tiles_x;                  /* tiles along x                       */
  long long units;              /* tiles * nz                          */
  int nblk;                     /* blocks; block b takes q or q+1 units */
  long long q, r;               /* units / nblk, units % nblk          */
  int gx, gy;                   /* staged passes: blocks work in groups
                                   of gx x gy neighbouring tiles (1 x 1
                                   elsewhere); q, r count group units  */
};

/* vector width usable for a row of nx cells of element size `esz` */
static int pick_vec(int nx, int esz)
{
  int v = 16 / esz;
  if(nx % (TX * v) == 0) return v;
  return 1;
}

static int sm_count(void)
{
  static int n = 0;
  if(!n) {
    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess ||
       cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess
       || n <= 0)
      n = 148;
  }
  return n;
}

/* `per_sm` resident blocks of the stencil kernels: the units are split
 * evenly over exactly one wave of resident blocks, so every SM holds the
 * same number of blocks (at least 4 planes per block) */
static boxc make_box(int nx, int ny, int nz, int perx, int pery, int perz,
  int dupx, int dupy, int dupz, int vec, int per_sm)
{
  boxc b;
  b.nx = nx; b.ny = ny; b.nz = nz;
  b.wW = perx ? (dupx ? nx - 2 : nx - 1) : 0;
  b.wE = perx ? (dupx ? 1 : 0) : nx - 1;
  b.wS = pery ? (dupy ? ny - 2 : ny - 1) : 0;
  b.wN = pery ? (dupy ? 1 : 0) : ny - 1;
  b.wB = perz ? (dupz ? nz - 2 : nz - 1) : 0;
  b.wT = perz ? (dupz ? 1 : 0) : nz - 1;
  b.vec = vec;
  b.gx = b.gy = 1;
  b.tiles_x = (nx + TX * vec - 1) / (TX * vec);
  long long tiles = (long long)b.tiles_x * ((ny + TY - 1) / TY);
  b.units = tiles * nz;
  if(per_sm < 1) per_sm = 1;
  long long slots = (long long)sm_count() * per_sm;
  long long nb = b.units / 4 < slots ? b.units / 4 : slots;
  if(nb < 1) nb = 1;
  b.nblk = (int)nb;
  b.q = b.units / nb;
  b.r = b.units % nb;
  return b;
}

static dim3 box_grid(const boxc &b)
{
  return dim3((unsigned)b.nblk);
}

template <typename K>
static int resident(K kernel)
{
  int nb = 0;
  if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, NTHR, 0)
     != cudaSuccess || nb < 1) {
    cudaGetLastError();
    nb = 2;
  }
  return nb;
}

__device__ __forceinline__ int mapx(const boxc &b, int g)
{ return g < 0 ? b.wW : (g >= b.nx ? (g == b.nx ? b.wE : b.nx - 1) : g); }
__device__ __forceinline__ int mapy(const boxc &b, int g)
{ return g < 0 ? b.wS : (g >= b.ny ? (g == b.ny ? b.wN : b.ny - 1) : g); }
__device__ __forceinline__ int mapz(const boxc &b, int g)
{ return g < 0 ? b.wB : (g >= b.nz ? (g == b.nz ? b.wT : b.nz - 1) : g); }

/* diagonal of the row with mask m, in the reference's summation order */
__host__ __device__ __forceinline__ double op_diag(unsigned m, const opc &O)
{
  if(m & BBB_MID) return 1.;
  double fW = (m & BBB_MW) ? 1. : 0., fE = (m & BBB_ME) ? 1. : 0.;
  double fS = (m & BBB_MS) ? 1. : 0., fN = (m & BBB_MN) ? 1. : 0.;
  double fB = (m & BBB_MB) ? 1. : 0., fT = (m & BBB_MT) ? 1. : 0.;
  if(!O.helm) {
    double d = 0.;
    d -= (fW + fE) * O.wx;
    d -= (fS + fN) * O.wy;
    d -= (fB + fT) * O.wz;
    return d;
  }
  double d = 1.;
  d += fW * O.wx; d += fE * O.wx;
  d += fS * O.wy; d += fN * O.wy;
  d += fB * O.wz; d += fT * O.wz;
  return d;
}

/* per-block tables of diagonal and Jacobi scale for the 128 mask bytes */
template <typename T>
struct optab {
  T diag[128];
  T dinv[128];
};

template <typename T>
__device__ __forceinline__ void optab_fill(optab<T> &t, const opc &O)
{
  int tid = threadIdx.x + blockDim.x * threadIdx.y;
  int nthr = blockDim.x * blockDim.y;
  for(int m = tid; m < 128; m += nthr) {
    double d = op_diag((unsigned)m, O);
    t.diag[m] = (T)d;
    t.dinv[m] = (T)(1. / d);
  }
  __syncthreads();
}

/* y = (A q)_c from the centre value, its six neighbours and the row mask;
 * neighbours in the order of the DIA diagonals: B, S, W, C, E, N, T */
template <typename T>
__device__ __forceinline__ T op_apply(unsigned m, const opc &O, T d, T qB,
  T qS, T qW, T qC, T qE, T qN, T qT)
{
  if(m & BBB_MID) return qC;
  T sg = O.helm ? (T)-1. : (T)1.;
  T wx = (T)O.wx * sg, wy = (T)O.wy * sg, wz = (T)O.wz * sg;
  T acc = (T)0.;
  acc += ((m & BBB_MB) ? wz : (T)0.) * qB;
  acc += ((m & BBB_MS) ? wy : (T)0.) * qS;
  acc += ((m & BBB_MW) ? wx : (T)0.) * qW;
  acc += d * qC;
  acc += ((m & BBB_ME) ? wx : (T)0.) * qE;
  acc += ((m & BBB_MN) ? wy : (T)0.) * qN;
  acc += ((m & BBB_MT) ? wz : (T)0.) * qT;
  return acc;
}

__device__ __forceinline__ long long lin(const boxc &b, int i, int j, int k)
{ return i + (long long)b.nx * (j + (long long)b.ny * k); }

/* ------------------------------------------------ vector access */
template <typename T, int V> struct VT;
template <> struct VT<float, 1> { typedef float t; };
template <> struct VT<float, 2> { typedef float2 t; };
template <> struct VT<float, 4> { typedef float4 t; };
template <> struct VT<double, 1> { typedef double t; };
template <> struct VT<double, 2> { typedef double2 t; };
template <int V> struct VM;
template <> struct VM<1> { typedef unsigned char t; };
template <> struct VM<2> { typedef uchar2 t; };
template <> struct VM<4> { typedef uchar4 t; };

template <typename T, int V>
__device__ __forceinline__ void ldv(const T *p, long long c, T (&o)[V])
{
  typename VT<T, V>::t x = *reinterpret_cast<const typename VT<T, V>::t *>(p + c);
  const T *e = reinterpret_cast<const T *>(&x);
#pragma unroll
  for(int v = 0; v < V; v++) o[v] = e[v];
}

template <typename T, int V>
__device__ __forceinline__ void stv(T *p, long long c, const T (&o)[V])
{
  typename VT<T, V>::t x;
  T *e = reinterpret_cast<T *>(&x);
#pragma unroll
  for(int v = 0; v < V; v++) e[v] = o[v];
  *reinterpret_cast<typename VT<T, V>::t *>(p + c) = x;
}

template <int V>
__device__ __forceinline__ void ldm(const uint8_t *p, long long c, unsigned (&o)[V])
{
  typename VM<V>::t x = *reinterpret_cast<const typename VM<V>::t *>(p + c);
  const unsigned char *e = reinterpret_cast<const unsigned char *>(&x);
#pragma unroll
  for(int v = 0; v < V; v++) o[v] = e[v];
}

/* the V mask bytes at c packed in one word (byte v = cell c + v) */
template <int V>
__device__ __forceinline__ unsigned ldmw(const uint8_t *p, long long c)
{
  if constexpr(V == 4) return *reinterpret_cast<const unsigned *>(p + c);
  else if constexpr(V == 2) return *reinterpret_cast<const unsigned short *>(p + c);
  else return p[c];
}

__device__ __forceinline__ unsigned mbyte(unsigned w, int v)
{ return (w >> (8 * v)) & 0xffu; }

/* two values carried from the producer to the epilogue */
template <typename T>
struct raw2 { T a, h; };

/* ------------------------------------------------ tiled stencil drivers
 * P: producer.  P::ev<V>(c, raw, q, dinv, own, red) gives at V consecutive
 * cells the value the operator is applied to (q) and what the epilogue
 * needs (raw, of type P::Raw); `own` is set exactly once for every cell of
 * the block's units, where the producer may also do the cell's
 * pointwise work (stores, sums into red).  E: epilogue; E::at<V>(c, raw,
 * Aq, red) at the owned cells, Aq = (A q) there. */

/* one cell per thread; any row length (partial tiles wrap by index);
 * planes k0..k1-1 of tile (bx, by) */
template <typename T, class P, class E, int NRED>
__device__ __forceinline__ void seg_stencil1(const boxc &B, const opc &O,
  const uint8_t *__restrict__ mask, const optab<T> &tab, P &prod, E &epi,
  double (&red)[NRED], int bx, int by, int k0, int k1)
{
  typedef typename P::Raw R;
  __shared__ T ring[3][HY][HX];
  int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
  int i0 = bx * TX, j0 = by * TY;
  int i = i0 + tx, j = j0 + ty;
  bool valid = (i < B.nx) && (j < B.ny);
  int gi = mapx(B, i), gj = mapy(B, j);
  int hsx = -1, hsy = -1, hgi = 0, hgj = 0;
  if(tid < 32) { hsx = tid + 1; hsy = 0; }
  else if(tid < 64) { hsx = tid - 32 + 1; hsy = HY - 1; }
  else if(tid < 72) { hsx = 0; hsy = tid - 64 + 1; }
  else if(tid < 80) { hsx = HX - 1; hsy = tid - 72 + 1; }
  if(hsx >= 0) { hgi = mapx(B, i0 - 1 + hsx); hgj = mapy(B, j0 - 1 + hsy); }

  R raw_cur[1], raw_next[1], hr[1];
  T q_prev[1], q_cur[1], q_next[1], hq[1];
  unsigned m_cur[1], m_next[1];
  prod.template ev<1>(lin(B, gi, gj, mapz(B, k0 - 1)), hr, q_prev, tab.dinv,
    false, red);
  {
    long long c = lin(B, gi, gj, k0);
    prod.template ev<1>(c, raw_cur, q_cur, tab.dinv, valid, red);
    ldm<1>(mask, c, m_cur);
    ring[0][ty + 1][tx + 1] = q_cur[0];
    if(hsx >= 0) {
      prod.template ev<1>(lin(B, hgi, hgj, k0), hr, hq, tab.dinv, false, red);
      ring[0][hsy][hsx] = hq[0];
    }
  }
  for(int k = k0; k < k1; k++) {
    int slot = (k - k0) % 3, nslot = (k - k0 + 1) % 3;
    long long cn = lin(B, gi, gj, mapz(B, k + 1));
    prod.template ev<1>(cn, raw_next, q_next, tab.dinv, valid && (k + 1 < k1),
      red);
    ldm<1>(mask, cn, m_next);
    if(k + 1 < k1) {
      ring[nslot][ty + 1][tx + 1] = q_next[0];
      if(hsx >= 0) {
        prod.template ev<1>(lin(B, hgi, hgj, k + 1), hr, hq, tab.dinv, false,
          red);
        ring[nslot][hsy][hsx] = hq[0];
      }
    }
    __syncthreads();
    if(valid) {
      T Aq[1];
      Aq[0] = op_apply<T>(m_cur[0], O, tab.diag[m_cur[0]], q_prev[0],
        ring[slot][ty][tx + 1], ring[slot][ty + 1][tx], q_cur[0],
        ring[slot][ty + 1][tx + 2], ring[slot][ty + 2][tx + 1], q_next[0]);
      epi.template at<1>(lin(B, i, j, k), raw_cur, Aq, red);
    }
    q_prev[0] = q_cur[0];
    raw_cur[0] = raw_next[0]; q_cur[0] = q_next[0];
    m_cur[0] = m_next[0];
  }
}

/* V cells per thread; requires nx % (32 V) == 0 (full tiles in x) */
template <typename T, int V, class P, class E, int NRED>
__device__ __forceinline__ void seg_stencilV(const boxc &B, const opc &O,
  const uint8_t *__restrict__ mask, const optab<T> &tab, P &prod, E &epi,
  double (&red)[NRED], int bx, int by, int k0, int k1)
{
  typedef typename P::Raw R;
  constexpr int W = TX * V;
  __shared__ __align__(16) T ring[3][HY][W];
  __shared__ T hw[3][TY], he[3][TY];
  int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
  int i0 = bx * W, j0 = by * TY;
  int ib = i0 + tx * V, j = j0 + ty;
  bool valid = j < B.ny;
  int gj = mapy(B, j);
  /* halo: two rows of W cells (vectors) and two columns of TY cells */
  int hrow = -1, hcol = -1, hgi = 0, hgj = 0;
  if(tid < 64) {
    hrow = tid < 32 ? 0 : HY - 1;
    hgi = i0 + (tid & 31) * V;
    hgj = mapy(B, hrow == 0 ? j0 - 1 : j0 + TY);
  } else if(tid < 80) {
    hcol = tid < 72 ? 0 : 1;
    int r = (tid - 64) & 7;
    hgi = mapx(B, hcol == 0 ? i0 - 1 : i0 + W);
    hgj = mapy(B, j0 + r);
  }
  R raw_cur[V], raw_next[V], tr[V];
  T q_prev[V], q_cur[V], q_next[V], tq[V];
  unsigned m_cur, m_next;
  prod.template ev<V>(lin(B, ib, gj, mapz(B, k0 - 1)), tr, q_prev, tab.dinv,
    false, red);
  {
    long long c = lin(B, ib, gj, k0);
    prod.template ev<V>(c, raw_cur, q_cur, tab.dinv, valid, red);
    m_cur = ldmw<V>(mask, c);
    stv<T, V>(&ring[0][ty + 1][0], tx * V, q_cur);
    if(hrow >= 0) {
      prod.template ev<V>(lin(B, hgi, hgj, k0), tr, tq, tab.dinv, false, red);
      stv<T, V>(&ring[0][hrow][0], (tid & 31) * V, tq);
    } else if(hcol >= 0) {
      R a[1];
      T bq[1];
      prod.template ev<1>(lin(B, hgi, hgj, k0), a, bq, tab.dinv, false, red);
      (hcol == 0 ? hw : he)[0][(tid - 64) & 7] = bq[0];
    }
  }
  for(int k = k0; k < k1; k++) {
    int slot = (k - k0) % 3, nslot = (k - k0 + 1) % 3;
    /* halo first: it only loads, so the owned cells' loads below can be
     * issued before its results are used */
    if(k + 1 < k1) {
      if(hrow >= 0) {
        prod.template ev<V>(lin(B, hgi, hgj, k + 1), tr, tq, tab.dinv, false,
          red);
        stv<T, V>(&ring[nslot][hrow][0], (tid & 31) * V, tq);
      } else if(hcol >= 0) {
        R a[1];
        T bq[1];
        prod.template ev<1>(lin(B, hgi, hgj, k + 1), a, bq, tab.dinv, false,
          red);
        (hcol == 0 ? hw : he)[nslot][(tid - 64) & 7] = bq[0];
      }
    }
    long long cn = lin(B, ib, gj, mapz(B, k + 1));
    prod.template ev<V>(cn, raw_next, q_next, tab.dinv, valid && (k + 1 < k1),
      red);
    m_next = ldmw<V>(mask, cn);
    if(k + 1 < k1) stv<T, V>(&ring[nslot][ty + 1][0], tx * V, q_next);
    __syncthreads();
    T left = __shfl_up_sync(0xffffffffu, q_cur[V - 1], 1);
    T right = __shfl_down_sync(0xffffffffu, q_cur[0], 1);
    if(tx == 0) left = hw[slot][ty];
    if(tx == TX - 1) right = he[slot][ty];
    if(valid) {
      T S[V], N[V], Aq[V];
      ldv<T, V>(&ring[slot][ty][0], tx * V, S);
      ldv<T, V>(&ring[slot][ty + 2][0], tx * V, N);
#pragma unroll
      for(int v = 0; v < V; v++) {
        T qW = v > 0 ? q_cur[v - 1] : left;
        T qE = v < V - 1 ? q_cur[v + 1] : right;
        unsigned mv = mbyte(m_cur, v);
        Aq[v] = op_apply<T>(mv, O, tab.diag[mv], q_prev[v], S[v], qW,
          q_cur[v], qE, N[v], q_next[v]);
      }
      epi.template at<V>(lin(B, ib, j, k), raw_cur, Aq, red);
    }
#pragma unroll
    for(int v = 0; v < V; v++) {
      q_prev[v] = q_cur[v];
      raw_cur[v] = raw_next[v]; q_cur[v] = q_next[v];
    }
    m_cur = m_next;
  }
}

/* this block's units, segment by segment (block-uniform loop) */
template <typename T, int V, class P, class E, int NRED>
__device__ __forceinline__ void tile_stencil(const boxc &B, const opc &O,
  const uint8_t *__restrict__ mask, const optab<T> &tab, P &prod, E &epi,
  double (&red)[NRED])
{
  long long bx_ = blockIdx.x;
  long long u0 = bx_ * B.q + (bx_ < B.r ? bx_ : B.r);
  long long u1 = u0 + B.q + (bx_ < B.r ? 1 : 0);
  while(u0 < u1) {
    long long tile = u0 / B.nz;
    int k0 = (int)(u0 - tile * B.nz);
    long long left = u1 - u0;
    int k1 = left < (long long)(B.nz - k0) ? k0 + (int)left : B.nz;
    int bx = (int)(tile % B.tiles_x), by = (int)(tile / B.tiles_x);
    if constexpr(V == 1)
      seg_stencil1<T>(B, O, mask, tab, prod, epi, red, bx, by, k0, k1);
    else
      seg_stencilV<T, V>(B, O, mask, tab, prod, epi, red, bx, by, k0, k1);
    u0 += k1 - k0;
    __syncthreads();      /* the ring is refilled by the next segment */
  }
}

/* ------------------------------------------------ masks */

/* Poisson rows: faces of cell (i,j,k) read at the reference's positions
 * (src/bicgstab_kernel.cu:1683-1716); identity where phase > -1
 * (src/bicgstab_kernel.cu:1826-1856) */
__global__ void k_mask_p(const int *fu, const int *fv, const int *fw,
  const int *phs, bbb_geom G, uint8_t *mask)
{
  long long n = (long long)G.nx * G.ny * G.nz;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx) + 1;
    long long r = t / G.nx;
    int j = (int)(r % G.ny) + 1, k = (int)(r / G.ny) + 1;
    long long W = i + (long long)j * G.fx_s1 + (long long)k * G.fx_s2;
    long long S = i + (long long)j * G.fy_s1 + (long long)k * G.fy_s2;
    long long Bq = i + (long long)j * G.fz_s1 + (long long)k * G.fz_s2;
    uint8_t m = 0;
    m |= fu[W] != 0 ? BBB_MW : 0;
    m |= fu[W + 1] != 0 ? BBB_ME : 0;
    m |= fv[S] != 0 ? BBB_MS : 0;
    m |= fv[S + G.fy_s1] != 0 ? BBB_MN : 0;
    m |= fw[Bq] != 0 ? BBB_MB : 0;
    m |= fw[Bq + G.fz_s2] != 0 ? BBB_MT : 0;
    if(phs[i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2] > -1) m |= BBB_MID;
    mask[t] = m;
  }
}

/* Helmholtz rows of component c on its face grid: face weights at the
 * mixed staggered positions the reference uses (src/bicgstab_kernel.cu:
 * 829-944), identity where the component's own flag < 0
 * (src/bicgstab_kernel.cu:730-827) */
/* the face (i, j, k) (1-based, ghosted grid) of dense index t of a
 * component system stored x-fastest in an X x Y x Z box, or, when `tr`,
 * y-fastest (the box's x axis is the grid's y axis) */
__device__ __forceinline__ void helm_ijk(long long t, int X, int Y, int tr,
  int &i, int &j, int &k)
{
  int a = (int)(t % X);
  long long r = t / X;
  int b = (int)(r % Y);
  k = (int)(r / Y) + 1;
  i = (tr ? b : a) + 1;
  j = (tr ? a : b) + 1;
}

/* dlo / dhi: the component's first / last face along its own axis is a
 * Dirichlet wall, whose rows are identity rows (the reference's
 * {u,v,w}star_coeffs_dirichlet_{W,E,S,N,B,T} for the wall normal to the
 * component, src/bicgstab_kernel.cu:946-1003, 1119-1176, 1291-1348; the
 * tangential walls' kernels zero couplings the face flags already drop) */
__global__ void k_mask_face(const int *fu, const int *fv, const int *fw,
  bbb_geom G, int comp, int nx, int ny, int nz, int tr, int dlo, int dhi,
  uint8_t *mask)
{
  long long n = (long long)nx * ny * nz;
  const int *fs = comp == 0 ? fu : (comp == 1 ? fv : fw);
  int s1 = comp == 0 ? G.fx_s1 : (comp == 1 ? G.fy_s1 : G.fz_s1);
  int s2 = comp == 0 ? G.fx_s2 : (comp == 1 ? G.fy_s2 : G.fz_s2);
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    helm_ijk(t, nx, ny, tr, i, j, k);
    long long W = i + (long long)j * G.fx_s1 + (long long)k * G.fx_s2;
    long long S = i + (long long)j * G.fy_s1 + (long long)k * G.fy_s2;
    long long Bq = i + (long long)j * G.fz_s1 + (long long)k * G.fz_s2;
    uint8_t m = 0;
    m |= fu[W] != 0 ? BBB_MW : 0;
    m |= fu[W + 1] != 0 ? BBB_ME : 0;
    m |= fv[S] != 0 ? BBB_MS : 0;
    m |= fv[S + G.fy_s1] != 0 ? BBB_MN : 0;
    m |= fw[Bq] != 0 ? BBB_MB : 0;
    m |= fw[Bq + G.fz_s2] != 0 ? BBB_MT : 0;
    if(fs[i + (long long)j * s1 + (long long)k * s2] < 0) m |= BBB_MID;
    const int a = comp == 0 ? i : (comp == 1 ? j : k);
    const int amax = comp == 0 ? G.nx + 1 : (comp == 1 ? G.ny + 1 : G.nz + 1);
    if((dlo && a == 1) || (dhi && a == amax)) m |= BBB_MID;
    if(tr) {
      /* the box's W/E faces are the grid's S/N and the other way round */
      uint8_t q = m & (BBB_MB | BBB_MT | BBB_MID);
      q |= (m & BBB_MS) ? BBB_MW : 0;
      q |= (m & BBB_MN) ? BBB_ME : 0;
      q |= (m & BBB_MW) ? BBB_MS : 0;
      q |= (m & BBB_ME) ? BBB_MN : 0;
      m = q;
    }
    mask[t] = m;
  }
}

/* the u system is stored y-fastest where its rows (nx + 1 faces) cannot
 * take the vector kernels and the grid's y rows can */
static int helm_tr(int comp, const bbb_geom &G)
{
  return comp == 0 && pick_vec(G.nx + 1, sizeof(float)) == 1
    && pick_vec(G.ny, sizeof(float)) == 4 && pick_vec(G.ny, sizeof(double)) == 2;
}

void bbb_build_masks(void)
{
  if(g_dev.masks_valid) return;
  bbb_geom G = bbb_make_geom();
  k_mask_p<<<NPW, 256, 0, g_dev.stream>>>(g_dev.flag_u, g_dev.flag_v,
    g_dev.flag_w, g_dev.phase, G, g_dev.mask_p);
  BBB_LAUNCHED();
  int tu = helm_tr(0, G);
  k_mask_face<<<NPW, 256, 0, g_dev.stream>>>(g_dev.flag_u, g_dev.flag_v,
    g_dev.flag_w, G, 0, tu ? G.ny : G.nx + 1, tu ? G.nx + 1 : G.ny, G.nz, tu,
    bc.uW == BBB_DIRICHLET, bc.uE == BBB_DIRICHLET, g_dev.mask_u);
  BBB_LAUNCHED();
  k_mask_face<<<NPW, 256, 0, g_dev.stream>>>(g_dev.flag_u, g_dev.flag_v,
    g_dev.flag_w, G, 1, G.nx, G.ny + 1, G.nz, 0,
    bc.vS == BBB_DIRICHLET, bc.vN == BBB_DIRICHLET, g_dev.mask_v);
  BBB_LAUNCHED();
  k_mask_face<<<NPW, 256, 0, g_dev.stream>>>(g_dev.flag_u, g_dev.flag_v,
    g_dev.flag_w, G, 2, G.nx, G.ny, G.nz + 1, 0,
    bc.wB == BBB_DIRICHLET, bc.wT == BBB_DIRICHLET, g_dev.mask_w);
  BBB_LAUNCHED();
  g_dev.masks_valid = 1;
}

/* ------------------------------------------------ BiCGSTAB kernels */

/* residual set-up: r = b - A x into s (pass A starts from r = s) and rh;
 * (r, r), sum x */
template <typename T>
struct prod_x {
  const T *x;
  typedef T Raw;
  template <int V, int NR>
  __device__ __forceinline__ void ev(long long c, T (&raw)[V], T (&q)[V],
    const T *dinv, bool own, double (&red)[NR]) const
  {
    ldv<T, V>(x, c, raw);
#pragma unroll
    for(int v = 0; v < V; v++) {
      q[v] = raw[v];
      if constexpr(NR > 1) { if(own) red[1] += (double)raw[v]; }
    }
    (void)dinv; (void)own;
  }
};
template <typename T>
struct epi_res {
  const T *b; T *r, *rh;
  template <int V>
  __device__ __forceinline__ void at(long long c, const T (&xr)[V],
    const T (&Ax)[V], double (&red)[2]) const
  {
    T bb[V], rv[V];
    ldv<T, V>(b, c, bb);
#pragma unroll
    for(int v = 0; v < V; v++) {
      rv[v] = bb[v] - Ax[v];
      red[0] += (double)rv[v] * (double)rv[v];
    }
    stv<T, V>(r, c, rv); stv<T, V>(rh, c, rv);
    (void)xr;
  }
};

template <typename T, int V>
__global__ void __launch_bounds__(NTHR) k_bicg_setup(boxc B, opc O,
  const uint8_t *__restrict__ mask, const T *__restrict__ b, const T *x,
  T *r0, T *rh, bbb_kry *s, double *partials, double rtol, int maxit)
{
  __shared__ double sh[32 * 2];
  __shared__ optab<T> tab;
  optab_fill<T>(tab, O);
  prod_x<T> P{x};
  epi_res<T> E{b, r0, rh};
  double red[2] = {0., 0.};
  tile_stencil<T, V>(B, O, mask, tab, P, E, red);
  if(bbb_grid_partial<2>(red, partials, &s->ticket, sh)) {
    bbb_grid_finish_sum<2>(red, partials, &s->ticket, sh);
    if(threadIdx.x == 0 && threadIdx.y == 0) {
      double rn = sqrt(red[0]);
      s->rho = red[0];
      s->rnorm = rn;
      s->tol = rtol * s->bnorm;
      s->sumx = red[1];
      s->iter = 0;
      s->maxit = maxit;
      s->first = 1;
      s->pad = 0;
      s->keep = 0;
      s->s_conv = 0;
      s->alpha = s->omega = s->beta = 0.;
      s->converged = (rn <= s->tol);
      s->done = s->converged || (maxit <= 0) || !isfinite(rn);
      s->status = isfinite(rn) ? 0 : BBB_ERR_NONFINITE;
    }
  }
}

/* pass A.  red: 0 (rh, v), 1 (r, r), 2 (rh, r), 3 sum x */
template <typename T>
struct prod_A {
  const T *s, *t, *p, *v, *rh; const uint8_t *mask;
  T *r_out, *p_out, *x;
  T alpha, omega, beta, bo;
  int first;
  typedef T Raw;                 /* rh at the cell */
  template <int V>
  __device__ __forceinline__ void ev(long long c, Raw (&raw)[V], T (&q)[V],
    const T *dinv, bool own, double (&red)[4]) const
  {
    T ss[V], rr[V], pn[V];
    unsigned mm[V];
    ldv<T, V>(s, c, ss);
    ldm<V>(mask, c, mm);
    if(first) {
#pragma unroll
      for(int a = 0; a < V; a++) { rr[a] = ss[a]; pn[a] = rr[a]; }
    } else {
      T tt[V], pp[V], vv[V];
      ldv<T, V>(t, c, tt);
      ldv<T, V>(p, c, pp);
      ldv<T, V>(v, c, vv);
#pragma unroll
      for(int a = 0; a < V; a++) {
        rr[a] = ss[a] - omega * tt[a];
        pn[a] = rr[a] + beta * pp[a] + bo * vv[a];
      }
      if(own) {
        T xx[V];
        ldv<T, V>(x, c, xx);
#pragma unroll
        for(int a = 0; a < V; a++) {
          T di = dinv[mm[a]];
          xx[a] = xx[a] + alpha * (di * pp[a]) + omega * (di * ss[a]);
          red[3] += (double)xx[a];
        }
        stv<T, V>(x, c, xx);
      }
    }
#pragma unroll
    for(int a = 0; a < V; a++) q[a] = dinv[mm[a]] * pn[a];
    if(own) {
      ldv<T, V>(rh, c, raw);
#pragma unroll
      for(int a = 0; a < V; a++) {
        red[1] += (double)rr[a] * (double)rr[a];
        red[2] += (double)raw[a] * (double)rr[a];
      }
      stv<T, V>(r_out, c, rr);
      stv<T, V>(p_out, c, pn);
    } else {
#pragma unroll
      for(int a = 0; a < V; a++) raw[a] = (T)0.;
    }
  }
};
template <typename T>
struct epi_A {
  T *vn;
  template <int V>
  __device__ __forceinline__ void at(long long c, const T (&hh)[V],
    const T (&Aq)[V], double (&red)[4]) const
  {
    stv<T, V>(vn, c, Aq);
#pragma unroll
    for(int a = 0; a < V; a++) red[0] += (double)hh[a] * (double)Aq[a];
  }
};

template <typename T, int V>
__global__ void __launch_bounds__(NTHR, BBB_KRY_MINB) k_bicgA(boxc B, opc O,
  const uint8_t *__restrict__ mask, const T *sv, const T *tv, const T *p_old,
  const T *v_old, const T *__restrict__ rh, T *r, T *p_new, T *v_new, T *x,
  bbb_kry *s, double *partials)
{
  if(((volatile bbb_kry *)s)->done) return;
  __shared__ double sh[32 * 4];
  __shared__ optab<T> tab;
  optab_fill<T>(tab, O);
  int first = s->first;
  double omega = s->omega, beta = s->beta;
  prod_A<T> P{sv, tv, p_old, v_old, rh, mask, r, p_new, x, (T)s->alpha,
    (T)omega, (T)beta, (T)(-beta * omega), first};
  epi_A<T> E{v_new};
  double red[4] = {0., 0., 0., 0.};
  tile_stencil<T, V>(B, O, mask, tab, P, E, red);
  if(bbb_grid_partial<4>(red, partials, &s->ticket, sh)) {
    bbb_grid_finish_sum<4>(red, partials, &s->ticket, sh);
    if(threadIdx.x == 0 && threadIdx.y == 0) {
      int sconv = s->s_conv;
      if(!first) {
        s->sumx = red[3];
        if(!sconv) s->iter += 1;
      }
      double rn = sconv ? s->rnorm : sqrt(red[1]);
      s->rnorm = rn;
      s->rho = red[2];
      s->rhv = red[0];
      s->alpha = red[2] / red[0];
      s->first = 0;
      s->converged = sconv || (rn <= s->tol);
      if(!isfinite(rn)) { s->status = BBB_ERR_NONFINITE; s->done = 1; }
      if(s->converged || s->iter >= s->maxit) s->done = 1;
      if(s->keep && !(rn <= 1e3 * s->rstart)) { s->status = -1; s->done = 1; }
    }
  }
}

/* pass B.  red: 0 (t, s), 1 (t, t), 2 (s, s), 3 (rh, s), 4 (rh, t) */
template <typename T>
struct prod_B {
  const T *r, *v; const uint8_t *mask; T *s_out; T alpha;
  typedef T Raw;                 /* s at the cell */
  template <int V>
  __device__ __forceinline__ void ev(long long c, T (&raw)[V], T (&q)[V],
    const T *dinv, bool own, double (&red)[5]) const
  {
    T rr[V], vv[V];
    unsigned mm[V];
    ldv<T, V>(r, c, rr);
    ldv<T, V>(v, c, vv);
    ldm<V>(mask, c, mm);
#pragma unroll
    for(int a = 0; a < V; a++) {
      raw[a] = rr[a] - alpha * vv[a];
      q[a] = dinv[mm[a]] * raw[a];
    }
    if(own) {
#pragma unroll
      for(int a = 0; a < V; a++) red[2] += (double)raw[a] * (double)raw[a];
      stv<T, V>(s_out, c, raw);
    }
  }
};
template <typename T>
struct epi_B {
  const T *rh; T *tn;
  template <int V>
  __device__ __forceinline__ void at(long long c, const T (&ss)[V],
    const T (&Aq)[V], double (&red)[5]) const
  {
    T hh[V];
    ldv<T, V>(rh, c, hh);
    stv<T, V>(tn, c, Aq);
#pragma unroll
    for(int a = 0; a < V; a++) {
      red[0] += (double)Aq[a] * (double)ss[a];
      red[1] += (double)Aq[a] * (double)Aq[a];
      red[3] += (double)hh[a] * (double)ss[a];
      red[4] += (double)hh[a] * (double)Aq[a];
    }
  }
};

template <typename T, int V>
__global__ void __launch_bounds__(NTHR, BBB_KRY_MINB) k_bicgB(boxc B, opc O,
  const uint8_t *__restrict__ mask, const T *r, const T *v,
  const T *__restrict__ rh, T *s_out, T *t_out, bbb_kry *s, double *partials)
{
  if(((volatile bbb_kry *)s)->done) return;
  __shared__ double sh[32 * 5];
  __shared__ optab<T> tab;
  optab_fill<T>(tab, O);
  double alpha = s->alpha;
  prod_B<T> P{r, v, mask, s_out, (T)alpha};
  epi_B<T> E{rh, t_out};
  double red[5] = {0., 0., 0., 0., 0.};
  tile_stencil<T, V>(B, O, mask, tab, P, E, red);
  if(bbb_grid_partial<5>(red, partials, &s->ticket, sh)) {
    bbb_grid_finish_sum<5>(red, partials, &s->ticket, sh);
    if(threadIdx.x == 0 && threadIdx.y == 0) {
      s->t_s = red[0];
      s->t_t = red[1];
      s->s_s = red[2];
      double sn = sqrt(red[2]);
      int sconv = (sn <= s->tol) && (!s->keep || sn == 0.);
      s->s_conv = sconv;
      if(sconv) {
        s->rnorm = sn;
        s->omega = 0.;
        s->beta = 0.;
      } else {
        double omega = red[0] / red[1];
        double rho_new = red[3] - omega * red[4];
        s->omega = omega;
        s->beta = (rho_new / s->rho) * (alpha / omega);
      }
    }
  }
}

#include "bbb_krylov_async.cuh"

/* ------------------------------------------------ Poisson set-up and
 * write-back (src/bicgstab_kernel.cu:483-562, src/particle_kernel.cu:
 * 840-940, src/cuda_bicgstab.cu:971-1045) */

/* b = rho_f/dt div(u*) in fluid cells, 0 in particle cells; x = phi;
 * ||b||^2 -> s->bnorm */
__global__ void k_pp_rhs(const real *us, const real *vs, const real *ws,
  const real *ph, const int *phs, bbb_geom G, double rho_dt, double *b,
  double *x, bbb_kry *s, double *partials)
{
  __shared__ double sh[32];
  double red[1] = {0.};
  long long n = (long long)G.nx * G.ny * G.nz;
  double ddx = 1. / G.dx, ddy = 1. / G.dy, ddz = 1. / G.dz;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx) + 1;
    long long rr = t / G.nx;
    int j = (int)(rr % G.ny) + 1, k = (int)(rr / G.ny) + 1;
    long long cu = i + (long long)j * G.fx_s1 + (long long)k * G.fx_s2;
    long long cv = i + (long long)j * G.fy_s1 + (long long)k * G.fy_s2;
    long long cw = i + (long long)j * G.fz_s1 + (long long)k * G.fz_s2;
    long long cc = i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2;
    double sv = (us[cu + 1] - us[cu]) * ddx;
    sv += (vs[cv + G.fy_s1] - vs[cv]) * ddy;
    sv += (ws[cw + G.fz_s2] - ws[cw]) * ddz;
    sv *= rho_dt;
    if(phs[cc] > -1) sv = 0.;
    b[t] = sv;
    x[t] = ph[cc];
    red[0] += sv * sv;
  }
  if(bbb_grid_partial<1>(red, partials, &s->ticket, sh)) {
    bbb_grid_finish_sum<1>(red, partials, &s->ticket, sh);
    if(threadIdx.x == 0) s->bnorm = sqrt(red[0]);
  }
}

__global__ void k_pp_writeback(const double *x, real *ph, bbb_geom G,
  const bbb_kry *s)
{
  long long n = (long long)G.nx * G.ny * G.nz;
  double mean = s->sumx / (double)n;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx) + 1;
    long long rr = t / G.nx;
    int j = (int)(rr % G.ny) + 1, k = (int)(rr / G.ny) + 1;
    ph[i + (long long)j * G.cc_s1 + (long long)k * G.cc_s2] = x[t] + -mean * 1.;
  }
}

/* ------------------------------------------------ live kernel timing
 * While enabled, CUDA events on the solver stream bracket each pass of
 * every BiCGSTAB iteration (slot 0: pass A, slot 1: pass B); after a solve
 * only the passes the device really executed are summed, each with its
 * algorithmic bytes (compulsory reads and writes of the owned cells). */
#define BBB_PROF_MAX 16384
#define BBB_PROF_SLOTS 6
static struct {
  int on, n;
  cudaEvent_t ev[2 * BBB_PROF_MAX];     /* start / end event of each launch */
  int slot[BBB_PROF_MAX];               /* BBB_PROF_* kind of the launch    */
  unsigned char ran[BBB_PROF_MAX];      /* 0: returned at once (after the
                                           solve had converged)            */
  double bytes[BBB_PROF_MAX];
  double ms[BBB_PROF_SLOTS], kbytes[BBB_PROF_SLOTS];
  long long launches[BBB_PROF_SLOTS];
  long long iters;
} g_prof;

/* before a launch: its slot and algorithmic bytes, start event */
static void prof_begin(int slot, double b)
{
  if(!g_prof.on || g_prof.n >= BBB_PROF_MAX) return;
  int i = g_prof.n;
  if(!g_prof.ev[2 * i]) cudaEventCreate(&g_prof.ev[2 * i]);
  if(!g_prof.ev[2 * i + 1]) cudaEventCreate(&g_prof.ev[2 * i + 1]);
  g_prof.slot[i] = slot;
  g_prof.bytes[i] = b;
  g_prof.ran[i] = 1;
  cudaEventRecord(g_prof.ev[2 * i], g_dev.stream);
}

/* after the launch: end event */
static void prof_end(void)
{
  if(!g_prof.on || g_prof.n >= BBB_PROF_MAX) return;
  cudaEventRecord(g_prof.ev[2 * g_prof.n + 1], g_dev.stream);
  g_prof.n++;
}

/* for launches made in the other source files (the momentum RHS) */
void bbb_prof_begin(int slot, double bytes) { prof_begin(slot, bytes); }
void bbb_prof_end(void) { prof_end(); }

/* index of the next record: the first launch of an iteration loop */
static int prof_mark(void) { return g_prof.on ? g_prof.n : 0; }

/* of the records from `from` on, only the first `nran` launches did work
 * (the device had converged before the later ones ran) */
static void prof_ran(int from, long long nran)
{
  if(!g_prof.on) return;
  for(int i = from; i < g_prof.n; i++)
    if(i - from >= nran) g_prof.ran[i] = 0;
}

/* the stream has been synchronised: sum the launches that did work */
static void prof_collect(void)
{
  if(!g_prof.on) return;
  for(int i = 0; i < g_prof.n; i++) {
    if(!g_prof.ran[i]) continue;
    float t = 0.f;
    if(cudaEventElapsedTime(&t, g_prof.ev[2 * i], g_prof.ev[2 * i + 1]) == cudaSuccess) {
      int sl = g_prof.slot[i];
      g_prof.ms[sl] += t;
      g_prof.kbytes[sl] += g_prof.bytes[i];
      g_prof.launches[sl]++;
    }
  }
  g_prof.n = 0;
}

extern "C" void bbb_profile_enable(int on) { g_prof.on = on; g_prof.n = 0; }
extern "C" void bbb_profile_reset(void)
{
  for(int a = 0; a < BBB_PROF_SLOTS; a++) {
    g_prof.ms[a] = 0.; g_prof.kbytes[a] = 0.; g_prof.launches[a] = 0;
  }
  g_prof.iters = 0; g_prof.n = 0;
}
extern "C" void bbb_profile_get(double *ms, long long *iters, double *bytes)
{
  *ms = 0.; *bytes = 0.;
  for(int a = 0; a < 2; a++) { *ms += g_prof.ms[a]; *bytes += g_prof.kbytes[a]; }
  *iters = g_prof.iters;
}
extern "C" void bbb_profile_get_pass(int pass, double *ms, long long *launches,
  double *bytes)
{
  if(pass < 0 || pass >= BBB_PROF_SLOTS) { *ms = 0.; *launches = 0; *bytes = 0.; return; }
  *ms = g_prof.ms[pass]; *launches = g_prof.launches[pass]; *bytes = g_prof.kbytes[pass];
}

/* the stage layout constants of one staged pass, in the order the header
 * lists them; host arithmetic only */
template <typename T, int PASS>
static int stage_layout(int *out, int nout)
{
  typedef as_layout<T, PASS> L;
  const int v[BBB_STAGE_LAYOUT_N] = {L::ESZ, L::CH, L::NA, L::NO, L::R, L::TH,
    L::WARPS, L::THREADS, L::BOXW, L::BOXH, L::ROWP, L::OWNB, L::EXT_OFF, L::AREG,
    L::MROWP, L::MEXT_OFF, L::MREG, L::MASK_OFF, L::OWN_OFF, L::XW_OFF, L::XWA,
    L::STAGE, L::NS, L::SMEM, L::TX_BASE, L::TX_XSIDE, L::TX_YSIDE, L::MINB};
  if(!out || nout < BBB_STAGE_LAYOUT_N) return -1;
  for(int a = 0; a < BBB_STAGE_LAYOUT_N; a++) out[a] = v[a];
  return BBB_STAGE_LAYOUT_N;
}

extern "C" int bbb_stage_layout(int fp64, int pass, int *out, int nout)
{
  if(fp64) {
    switch(pass) {
    case 0: return stage_layout<double, 0>(out, nout);
    case 1: return stage_layout<double, 1>(out, nout);
    case 2: return stage_layout<double, 2>(out, nout);
    case 3: return stage_layout<double, 3>(out, nout);
    }
  } else {
    switch(pass) {
    case 0: return stage_layout<float, 0>(out, nout);
    case 1: return stage_layout<float, 1>(out, nout);
    case 3: return stage_layout<float, 3>(out, nout);
    }
  }
  return -1;
}

/* run iterations until the device says done; the host polls the scalars
 * in growing batches so a converged solve costs at most a few no-op
 * launches */
template <typename LaunchIter>
static int drive(bbb_kry *s, LaunchIter launch_iter, int maxit, int batch0)
{
  int batch = batch0, total = 0;
  for(;;) {
    for(int q = 0; q < batch; q++) launch_iter();
    total += batch;
    BBB_CK(cudaMemcpyAsync(g_dev.kry_host, s, sizeof(bbb_kry),
      cudaMemcpyDeviceToHost, g_dev.stream));
    BBB_CK(cudaStreamSynchronize(g_dev.stream));
    if(bbb_last_status() == BBB_ERR_CUDA) return -1;
    if(g_dev.kry_host->done) break;
    if(total > maxit + 4) break;
    if(batch < 16) batch *= 2;
  }
  return g_dev.kry_host->iter;
}

/* resident blocks per SM of the two passes of precision T and width V */
template <typename T, int V>
static int bicg_per_sm(void)
{
  static int nb = 0;
  if(!nb) {
    int a = resident(k_bicgA<T, V>), b = resident(k_bicgB<T, V>);
    nb = a < b ? a : b;
  }
  return nb;
}

/* resident blocks per SM of the staged passes (0 when they cannot run) */
template <typename T, int PASS>
static int as_per_sm(void)
{
  static int nb = -1;
  if(nb < 0) {
    typedef as_layout<T, PASS> L;
    nb = 0;
    if(cudaFuncSetAttribute(k_bicg_async<T, PASS>,
         cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM) == cudaSuccess) {
      int v = 0;
      if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_bicg_async<T, PASS>,
           L::THREADS, L::SMEM) == cudaSuccess) nb = v;
    }
    cudaGetLastError();
  }
  return nb;
}

/* The same box cut into 128-cell tiles for a kernel with `per_sm`
 * resident blocks, in groups of gx x gy neighbouring tiles.  A group's
 * blocks take the same run of planes, one tile each, so every tile's x and
 * y neighbours inside the group are read at the same planes at the same
 * time and the halo rows and chunks they share come from L2, not DRAM; the
 * group units (group, plane) are split evenly over one wave of groups
 * (gx = tiles_x when the rows hold at most two tiles, gy = 4 or 2 where the
 * tile rows and the slots divide).  On 256x256x512 in FP32 this took pass
 * A's DRAM reads from 1.78x to 1.07x its algorithmic reads and the launch
 * from 0.36 to 0.26 ms.  `align` additionally cuts every group's planes
 * into equal runs so that all groups start at the same planes, where at
 * least 80% of the slots stay busy (slower than grouping alone there). */
static boxc retile(const boxc &B0, int per_sm, bool align, int th = 8, int gxw = 0,
  int gyw = 0)
{
  boxc b = B0;
  b.vec = AS_W / TX;
  b.tiles_x = b.nx / AS_W;
  int tiles_y = (b.ny + th - 1) / th;
  long long all = (long long)sm_count() * (per_sm > 0 ? per_sm : 1);
  int gx = gxw > 0 ? gxw : (b.tiles_x <= 2 ? b.tiles_x : 1);
  if(b.tiles_x % gx) gx = 1;
  /* the tallest group (4, 2, 1 tiles) that divides the tile rows and
   * leaves no resident slot idle */
  int gy = gyw;
  if(gy <= 0)
    for(gy = 4; gy > 1; gy /= 2)
      if(tiles_y % gy == 0 && tiles_y >= 4 * gy && all % (gx * gy) == 0) break;
  if(tiles_y % gy) gy = 1;
  b.gx = gx; b.gy = gy;
  long long G = (long long)gx * gy;
  long long groups = (long long)(b.tiles_x / gx) * (tiles_y / gy);
  long long gunits = groups * b.nz;
  b.units = gunits * G;
  long long slots = all / G;
  if(slots < 1) slots = 1;
  long long ng = gunits / 4 < slots ? gunits / 4 : slots;
  if(align) {
    long long m = slots / groups;
    while(m > 1 && b.nz / m < 4) m--;
    if(m >= 1 && groups * m * 5 >= slots * 4) ng = groups * m;
  }
  if(ng < 1) ng = 1;
  b.nblk = (int)(ng * G);
  b.q = gunits / ng;
  b.r = gunits % ng;
  return b;
}

/* cuTensorMapEncodeTiled through the CUDA runtime's driver entry point (no
 * link against libcuda); NULL when the installed CUDA driver lacks it */
typedef CUresult (*as_encode_fn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t,
  void *, const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static as_encode_fn as_encoder(void)
{
  static as_encode_fn f = NULL;
  static int tried = 0;
  if(!tried) {
    tried = 1;
    void *p = NULL;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q)
         == cudaSuccess && q == cudaDriverEntryPointSuccess)
      f = (as_encode_fn)p;
    cudaGetLastError();
  }
  return f;
}

/* map of a dense nx*ny*nz array of `esz`-byte elements (8: FP64, 4: FP32,
 * 1: mask bytes) read in boxes of {bx, by, 1}; out-of-range cells read 0 */
static bool as_map(CUtensorMap *m, const void *base, int esz, const boxc &B,
  int bx, int by)
{
  as_encode_fn enc = as_encoder();
  if(!enc || !base) return false;
  CUtensorMapDataType dt = esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
    : (esz == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT8);
  cuuint64_t dim[3] = {(cuuint64_t)B.nx, (cuuint64_t)B.ny, (cuuint64_t)B.nz};
  cuuint64_t str[2] = {(cuuint64_t)B.nx * esz, (cuuint64_t)B.nx * B.ny * esz};
  cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  cuuint32_t es[3] = {1, 1, 1};
  return enc(m, dt, 3, const_cast<void *>(base), dim, str, box, es,
    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)
    == CUDA_SUCCESS;
}

/* the maps of one staged pass: halo arrays h[0..na), own arrays o[0..no) */
template <typename T, int PASS>
static bool as_pass_maps(as_maps *M, const boxc &B, const uint8_t *mask,
  const T *const *h, const T *const *o)
{
  typedef as_layout<T, PASS> L;
  memset(M, 0, sizeof(*M));
  bool ok = as_map(&M->m, mask, 1, B, L::MBOXW, L::BOXH)
    && as_map(&M->mx, mask, 1, B, 16, L::TH);
  for(int a = 0; a < L::NA && ok; a++)
    ok = as_map(&M->h[a], h[a], L::ESZ, B, L::BOXW, L::BOXH)
      && as_map(&M->hx[a], h[a], L::ESZ, B, L::CH, L::TH);
  for(int b = 0; b < L::NO && ok; b++)
    ok = as_map(&M->o[b], o[b], L::ESZ, B, AS_W, L::TH);
  return ok;
}

/* the staged passes run where rows are a multiple of 128 cells */
#ifndef BBB_NO_ASYNC
#define BBB_ASYNC_ON 1
#else
#define BBB_ASYNC_ON 0
#endif

/* BiCGSTAB iterations after a set-up kernel.  Fresh (`resume` false): the
 * set-up left s = r0 = rh and first = 1; launches go A, B, A, B, ...
 * Resumed after a residual replacement: r holds the replaced residual,
 * alpha its (rh, r) / (rh, v), p and v the directions in buffers *curp;
 * launches go B, A, B, A, ...  Either way a run ends after a pass A.
 * *curp (when given) returns the buffer index of the latest p, v. */
template <typename T, int V>
static void bicgstab_iterations(const boxc &B, const opc &O, long long n,
  const uint8_t *mask, T *r, T *rh, T *p0, T *p1, T *v0, T *v1, T *sv, T *tv,
  T *x, bbb_kry *s, int maxit, int batch0, int *curp = NULL, bool resume = false)
{
  dim3 grd = box_grid(B), blk(TX, TY);
  T *pp[2] = {p0, p1}, *vv[2] = {v0, v1};
  const int cur0 = curp ? *curp : 0;
  int cur = cur0, launched = 0;
  double w = sizeof(T);
  bool staged = BBB_ASYNC_ON && B.nx % AS_W == 0 && as_per_sm<T, 0>() > 0
    && as_per_sm<T, 1>() > 0;
  boxc BA = B, BB = B;
  /* The staged passes keep r in two buffers, rr[0] = sv and rr[1] = r:
   * pass A reads r from rr[rc] and writes the new r to rr[rc ^ 1], and
   * pass B, which stores no s, reads r from rr[rc].  A fresh solve's
   * set-up leaves s = r0 in sv, which the opening pass A reads as its r
   * (rc = 0); a resumed run starts with pass B on the replaced residual
   * the set-up wrote to r (rc = 1). */
  T *rr[2] = {sv, r};
  int rc = resume ? 1 : 0;
  as_maps MA[2][2], MB[2][2];   /* [r buffer][p, v buffer] */
  if(staged) {
    BA = retile(B, as_per_sm<T, 0>(), as_layout<T, 0>::ALIGN, as_layout<T, 0>::TH);
    BB = retile(B, as_per_sm<T, 1>(), as_layout<T, 1>::ALIGN, as_layout<T, 1>::TH);
    for(int q = 0; q < 2 && staged; q++)
      for(int c = 0; c < 2 && staged; c++) {
        const T *ha[4] = {rr[q], tv, pp[c], vv[c]}, *oa[2] = {x, rh};
        const T *hb[4] = {rr[q], vv[c], NULL, NULL}, *ob[2] = {rh, NULL};
        staged = as_pass_maps<T, 0>(&MA[q][c], BA, mask, ha, oa)
              && as_pass_maps<T, 1>(&MB[q][c], BB, mask, hb, ob);
      }
  }
  /* pass A: reads p, v of buffer cur, writes buffer cur ^ 1, then cur flips
   * (and, staged, the r buffer with it) */
  auto pass_a = [&]() {
    /* the opening pass of a fresh solve reads s, rh; later ones s (staged:
     * r), t, p, v, x, rh; + mask */
    double a_bytes = (launched == 0 && !resume) ? (double)n * (5. * w + 1.)
                                                : (double)n * (10. * w + 1.);
    prof_begin(BBB_PROF_PASS_A, a_bytes);
    if(staged) {
      as_args<T> A = {};
      A.mask = mask;
      A.h[0] = rr[rc]; A.h[1] = tv; A.h[2] = pp[cur]; A.h[3] = vv[cur];
      A.w0 = rr[rc ^ 1]; A.w1 = pp[cur ^ 1]; A.w2 = vv[cur ^ 1]; A.x = x;
      A.s = s; A.partials = g_dev.partials;
      k_bicg_async<T, 0><<<BA.nblk, as_layout<T, 0>::THREADS, as_layout<T, 0>::SMEM,
        g_dev.stream>>>(BA, O, A, MA[rc][cur]);
      rc ^= 1;
    } else {
      k_bicgA<T, V><<<grd, blk, 0, g_dev.stream>>>(B, O, mask, sv, tv, pp[cur],
        vv[cur], rh, r, pp[cur ^ 1], vv[cur ^ 1], x, s, g_dev.partials);
    }
    BBB_LAUNCHED();
    prof_end();
    cur ^= 1;
    launched++;
  };
  /* pass B: reads r and the latest v (buffer cur); staged, it writes t
   * only (4 words + mask per unknown), else s and t */
  auto pass_b = [&]() {
    prof_begin(BBB_PROF_PASS_B, (double)n * ((staged ? 4. : 5.) * w + 1.));
    if(staged) {
      as_args<T> A = {};
      A.mask = mask;
      A.h[0] = rr[rc]; A.h[1] = vv[cur]; A.h[2] = NULL; A.h[3] = NULL;
      A.w0 = NULL; A.w1 = tv; A.w2 = NULL; A.x = NULL;
      A.s = s; A.partials = g_dev.partials;
      k_bicg_async<T, 1><<<BB.nblk, as_layout<T, 1>::THREADS, as_layout<T, 1>::SMEM,
        g_dev.stream>>>(BB, O, A, MB[rc][cur]);
    } else {
      k_bicgB<T, V><<<grd, blk, 0, g_dev.stream>>>(B, O, mask, r, vv[cur],
        rh, sv, tv, s, g_dev.partials);
    }
    BBB_LAUNCHED();
    prof_end();
  };
  const int pmark = prof_mark();
  if(resume) drive(s, [&]() { pass_b(); pass_a(); }, maxit, batch0);
  else drive(s, [&]() { pass_a(); pass_b(); }, maxit, batch0);
  /* passes executed -- fresh: the opening pass A, B and A of each counted
   * iteration, B and A of an uncounted one that ended on ||s|| (a solve
   * that converged at set-up ran none); resumed: B and A of each counted
   * iteration and of an uncounted last one */
  bbb_kry *h = g_dev.kry_host;
  long long npass;
  if(resume) npass = 2LL * h->iter + (h->s_conv ? 2 : 0);
  else npass = h->first ? 0 : 2LL * h->iter + 1 + (h->s_conv ? 2 : 0);
  prof_ran(pmark, npass);
  if(g_prof.on) g_prof.iters += npass / 2;
  prof_collect();
  /* launches after convergence return at once but still flip `cur`: the
   * latest p, v are where the passes A that really ran left them */
  if(curp) {
    long long na = resume ? h->iter + (h->s_conv ? 1 : 0)
                          : (h->first ? 0 : 1 + h->iter + (h->s_conv ? 1 : 0));
    *curp = cur0 ^ (int)(na & 1);
  }
}

static opc poisson_op(const bbb_geom &G)
{
  opc O;
  O.wx = 1. / (G.dx * G.dx); O.wy = 1. / (G.dy * G.dy); O.wz = 1. / (G.dz * G.dz);
  O.helm = 0;
  return O;
}

template <int V>
static void poisson_fp64(const boxc &B, const opc &O, long long n, bbb_kry *s)
{
  dim3 grd = box_grid(B), blk(TX, TY);
  k_bicg_setup<double, V><<<grd, blk, 0, g_dev.stream>>>(B, O, g_dev.mask_p,
    g_dev.kb, g_dev.kx, g_dev.ks, g_dev.krh, s, g_dev.partials, bbb_pp_tol(),
    pp_max_iter);
  BBB_LAUNCHED();
  bicgstab_iterations<double, V>(B, O, n, g_dev.mask_p, g_dev.kr, g_dev.krh,
    g_dev.kp[0], g_dev.kp[1], g_dev.kv[0], g_dev.kv[1], g_dev.ks, g_dev.kt,
    g_dev.kx, s, pp_max_iter, 1);
}

int bbb_poisson_solve(int record)
{
  bbb_dev_require();
  if(!g_dev.ready) return -1;
  bbb_build_masks();
  bbb_geom G = bbb_make_geom();
  int V = pick_vec(G.nx, sizeof(double));
  int per_sm = V == 2 ? bicg_per_sm<double, 2>() : bicg_per_sm<double, 1>();
  boxc B = make_box(G.nx, G.ny, G.nz, bc.pW == BBB_PERIODIC,
    bc.pS == BBB_PERIODIC, bc.pB == BBB_PERIODIC, 0, 0, 0, V, per_sm);
  opc O = poisson_op(G);
  long long n = (long long)G.nx * G.ny * G.nz;
  bbb_kry *s = g_dev.kry;
  k_pp_rhs<<<NPW, 256, 0, g_dev.stream>>>(g_dev.us, g_dev.vs, g_dev.ws,
    g_dev.phi, g_dev.phase, G, rho_f / dt, g_dev.kb, g_dev.kx, s, g_dev.partials);
  BBB_LAUNCHED();
  bbb_learn_pre_solve();
  if(V == 2) poisson_fp64<2>(B, O, n, s);
  else poisson_fp64<1>(B, O, n, s);
  k_pp_writeback<<<NPW, 256, 0, g_dev.stream>>>(g_dev.kx, g_dev.phi, G, s);
  BBB_LAUNCHED();
  bbb_learn_post_solve();
  BBB_CK(cudaMemcpyAsync(g_dev.kry_host, s, sizeof(bbb_kry),
    cudaMemcpyDeviceToHost, g_dev.stream));
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
  bbb_kry *h = g_dev.kry_host;
  real resid = h->bnorm > 0 ? h->rnorm / h->bnorm : h->rnorm;
  if(g_stats.pp_solves == 0) g_stats.pp_iters_first = h->iter;
  g_stats.pp_solves++;
  g_stats.pp_iters_total += h->iter;
  g_stats.pp_iters_last = h->iter;
  if(h->iter > g_stats.pp_iters_max) g_stats.pp_iters_max = h->iter;
  g_stats.pp_resid_last = resid;
  g_stats.pp_outer_last = 1;
  bbb_learn_solve_done(h->rnorm);
  if(record) bbb_record_solver("solver_expd.rec", h->iter, resid);
  if(h->status == BBB_ERR_NONFINITE) bbb_set_status(BBB_ERR_NONFINITE, "pressure-Poisson");
  if(!h->converged) {
    bbb_set_status(BBB_ERR_NOT_CONVERGED, "pressure-Poisson");
    if(bbb_fail_exit()) {
      printf("The pressure-Poisson equation did not converge.              \n");
      exit(EXIT_FAILURE);
    }
  }
  return h->iter;
}

/* ------------------------------------------------ mixed precision
 * Defect correction: the FP64 outer loop forms r = b - A x in FP64 (with
 * ||r||, the stopping test of the FP64 form, and sum x for the mean),
 * hands r to an FP32 Jacobi-BiCGSTAB that solves A e = r from e = 0, and
 * accumulates x += e in FP64.  The inner target is `inner_tol` relative,
 * or looser when half the remaining reduction already meets the outer
 * test.  Stops when the FP64 residual meets pp_residual * ||b||, the same
 * test as the FP64 form.  Without particle rows the periodic/Neumann
 * operator is singular; the inner right-hand side is then projected onto
 * zero mean. */

struct epi_res64 {
  const double *b; float *rf;
  template <int V>
  __device__ __forceinline__ void at(long long c, const double (&xr)[V],
    const double (&Ax)[V], double (&red)[3]) const
  {
    double bb[V];
    ldv<double, V>(b, c, bb);
#pragma unroll
    for(int a = 0; a < V; a++) {
      double rv = bb[a] - Ax[a];
      rf[c + a] = (float)rv;
      red[0] += rv * rv;
      red[2] += rv;
    }
    (void)xr;
  }
};

/* outer residual; the finaliser decides convergence and sets up the inner
 * solve's tolerance */
template <int V>
__global__ void __launch_bounds__(NTHR) k_outer_resid(boxc B, opc O,
  const uint8_t *__restrict__ mask, const double *__restrict__ b,
  const double *x, float *rf, bbb_kry *s, bbb_kry *si, double *partials,
  double inner_tol, int inner_maxit, int project_mean, long long n)
{
  __shared__ double sh[32 * 3];
  __shared__ optab<double> tab;
  optab_fill<double>(tab, O);
  prod_x<double> P{x};
  epi_res64 E{b, rf};
  double red[3] = {0., 0., 0.};
  tile_stencil<double, V>(B, O, mask, tab, P, E, red);
  if(bbb_grid_partial<3>(red, partials, &s->ticket, sh)) {
    bbb_grid_finish_sum<3>(red, partials, &s->ticket, sh);
    if(threadIdx.x == 0 && threadIdx.y == 0) {
      double rn = sqrt(red[0]);
      s->rnorm = rn;
      s->sumx = red[1];
      s->converged = (rn <= s->tol);
      s->s_conv = 0;
      if(!isfinite(rn)) { s->status = BBB_ERR_NONFINITE; s->done = 1; }
      if(s->converged || s->iter >= s->maxit) s->done = 1;
      double mean = project_mean ? red[2] / (double)n : 0.;
      si->sumx = mean;                 /* subtracted by the inner set-up */
      double need = rn > 0. ? 0.5 * s->tol / rn : 1.;
      si->tol = fmax(inner_tol, need) * rn;
      si->maxit = inner_maxit;
      si->done = s->done;
      if(s->done) {
        /* no inner sweep follows: it reports no iterations or passes */
        si->iter = 0; si->first = 1; si->s_conv = 0;
      }
    }
  }
}

/* inner set-up from e = 0: s = rh = rf - mean (pass A starts from r = s),
 * e = 0, (r, r) */
template <int V>
__global__ void __launch_bounds__(256) k_inner_setup(long long n,
  const float *__restrict__ rf, float *s0, float *e, float *rh, bbb_kry *si,
  double *partials)
{
  if(((volatile bbb_kry *)si)->done) return;
  __shared__ double sh[32];
  float mean = (float)si->sumx;
  double red[1] = {0.};
  long long nv = n / V;
  for(long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nv;
      q += (long long)gridDim.x * blockDim.x) {
    long long c = q * V;
    float rv[V], z[V];
    ldv<float, V>(rf, c, rv);
#pragma unroll
    for(int a = 0; a < V; a++) {
      rv[a] = rv[a] - mean;
      z[a] = 0.f;
      red[0] += (double)rv[a] * (double)rv[a];
    }
    stv<float, V>(s0, c, rv); stv<float, V>(rh, c, rv);
    stv<float, V>(e, c, z);
  }
  if(bbb_grid_partial<1>(red, partials, &si->ticket, sh)) {
    bbb_grid_finish_sum<1>(red, partials, &si->ticket, sh);
    if(threadIdx.x == 0) {
      double rn = sqrt(red[0]);
      si->rho = red[0];
      si->rnorm = rn;
      si->iter = 0;
      si->first = 1;
      si->pad = 0;
      si->keep = 1;
      si->rstart = INFINITY;
      si->s_conv = 0;
      si->alpha = si->omega = si->beta = 0.;
      si->converged = (rn <= si->tol);
      si->done = si->converged || si->maxit <= 0 || !isfinite(rn);
      si->status = isfinite(rn) ? 0 : BBB_ERR_NONFINITE;
    }
  }
}

/* Residual replacement inside a running inner solve (reliable update):
 * r = rf - mean (rf the FP64 residual b - A x of the accumulated solution,
 * rounded to FP32), e = 0; the Krylov state p, v, rh stays.  rho = (rh, r)
 * and alpha = rho / (rh, v) restart the recurrences from the true residual
 * -- the group-wise residual replacement of Sleijpen and van der Vorst
 * ("Reliable updated residuals in hybrid Bi-CG methods", Computing 56,
 * 1996), which keeps the FP32 recursion's residual gap below what the
 * FP64 stopping test needs without discarding the Krylov space. */
template <int V>
__global__ void __launch_bounds__(256) k_reliable_setup(long long n,
  const float *__restrict__ rf, const float *__restrict__ rh, float *r, float *e,
  bbb_kry *si, double *partials)
{
  if(((volatile bbb_kry *)si)->done) return;
  __shared__ double sh[32 * 2];
  float mean = (float)si->sumx;
  double red[2] = {0., 0.};
  long long nv = n / V;
  for(long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nv;
      q += (long long)gridDim.x * blockDim.x) {
    long long c = q * V;
    float rv[V], hv[V], z[V];
    ldv<float, V>(rf, c, rv);
    ldv<float, V>(rh, c, hv);
#pragma unroll
    for(int a = 0; a < V; a++) {
      rv[a] = rv[a] - mean;
      z[a] = 0.f;
      red[0] += (double)rv[a] * (double)rv[a];
      red[1] += (double)hv[a] * (double)rv[a];
    }
    stv<float, V>(r, c, rv);
    stv<float, V>(e, c, z);
  }
  if(bbb_grid_partial<2>(red, partials, &si->ticket, sh)) {
    bbb_grid_finish_sum<2>(red, partials, &si->ticket, sh);
    if(threadIdx.x == 0) {
      double rn = sqrt(red[0]);
      si->rnorm = rn;
      si->rho = red[1];
      si->alpha = red[1] / si->rhv;
      si->iter = 0;
      si->first = 0;
      si->pad = 0;
      si->keep = 1;
      si->rstart = rn;
      si->s_conv = 0;
      si->converged = (rn <= si->tol);
      si->done = si->converged || si->maxit <= 0 || !isfinite(rn)
        || !isfinite(si->alpha);
      si->status = isfinite(rn) && isfinite(si->alpha) ? 0 : BBB_ERR_NONFINITE;
    }
  }
}

/* x += e */
template <int V>
__global__ void __launch_bounds__(256) k_accumulate(long long n, double *x,
  const float *__restrict__ e, bbb_kry *s)
{
  if(((volatile bbb_kry *)s)->done) return;
  long long nv = n / V;
  for(long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nv;
      q += (long long)gridDim.x * blockDim.x) {
    long long c = q * V;
    float ev_[V];
    ldv<float, V>(e, c, ev_);
#pragma unroll
    for(int a = 0; a < V; a++) x[c + a] = x[c + a] + (double)ev_[a];
  }
  if(blockIdx.x == 0 && threadIdx.x == 0) s->iter += 1;   /* outer sweeps */
}

static void ensure_fp32(void)
{
  if(g_dev.fb) return;
  long long n = g_dev.nmax;
  float **fs[] = {&g_dev.fb, &g_dev.fx, &g_dev.fr, &g_dev.frh, &g_dev.fp[0],
    &g_dev.fp[1], &g_dev.fv[0], &g_dev.fv[1], &g_dev.fs, &g_dev.ft};
  for(size_t a = 0; a < sizeof(fs) / sizeof(fs[0]); a++) {
    if(cudaMalloc((void **)fs[a], sizeof(float) * (size_t)n) != cudaSuccess)
      bbb_set_status(BBB_ERR_CUDA, "cudaMalloc fp32 workspace");
    else
      cudaMemsetAsync(*fs[a], 0, sizeof(float) * (size_t)n, g_dev.stream);
  }
  if(!g_dev.kry_inner) {
    if(cudaMalloc((void **)&g_dev.kry_inner, sizeof(bbb_kry)) != cudaSuccess)
      bbb_set_status(BBB_ERR_CUDA, "cudaMalloc inner scalars");
    cudaMemsetAsync(g_dev.kry_inner, 0, sizeof(bbb_kry), g_dev.stream);
  }
}

/* The FP64 outer residual of a defect-correction sweep, r = b - A x into
 * FP32 rf with the sweep's scalars: the tensor-map staged pass where the
 * rows are a multiple of 128 cells, else the register-tiled kernel. */
template <int VD>
static void outer_resid(const boxc &BD, const opc &O, const uint8_t *mask,
  const double *b, const double *x, float *rf, bbb_kry *s, bbb_kry *si,
  double itol, int imaxit, int project, long long n)
{
  if(BBB_ASYNC_ON && BD.nx % AS_W == 0 && as_per_sm<double, 2>() > 0) {
    boxc B2 = retile(BD, as_per_sm<double, 2>(), false, as_layout<double, 2>::TH);
    as_maps M;
    const double *h[4] = {x, NULL, NULL, NULL}, *o[2] = {b, NULL};
    if(as_pass_maps<double, 2>(&M, B2, mask, h, o)) {
      as_args<double> A;
      memset(&A, 0, sizeof(A));
      A.mask = mask; A.h[0] = x; A.s = s; A.partials = g_dev.partials;
      A.rf = rf; A.si = si; A.itol = itol; A.imaxit = imaxit;
      A.project = project; A.n = n;
      prof_begin(BBB_PROF_OUTER, (double)n * (2. * 8. + 4. + 1.));
      k_bicg_async<double, 2><<<B2.nblk, as_layout<double, 2>::THREADS,
        as_layout<double, 2>::SMEM,
        g_dev.stream>>>(B2, O, A, M);
      BBB_LAUNCHED();
      prof_end();
      return;
    }
  }
  dim3 grd = box_grid(BD), blk(TX, TY);
  prof_begin(BBB_PROF_OUTER, (double)n * (2. * 8. + 4. + 1.));
  k_outer_resid<VD><<<grd, blk, 0, g_dev.stream>>>(BD, O, mask, b, x, rf, s, si,
    g_dev.partials, itol, imaxit, project, n);
  BBB_LAUNCHED();
  prof_end();
}

/* Fail-fast rule of a defect-correction solve.  The inner iterations of all
 * sweeps share one budget, pp_max_iter -- the cap of the whole FP64 solve,
 * as CUSP's monitor caps the reference's (src/cuda_bicgstab.cu:996-1018) --
 * and the FP64 residual must halve at least every two sweeps.  A solve that
 * breaks either rule stops at once as not converged, so a diverging or
 * stagnating solve reports after at most pp_max_iter inner iterations
 * instead of running every sweep to its own cap. */
struct dc_guard {
  int budget, used, sweeps;
  double hist[2];                 /* FP64 ||r|| of the two previous sweeps */
  explicit dc_guard(int b) : budget(b), used(0), sweeps(0) { hist[0] = hist[1] = -1.; }
  int remaining() const { return budget - used; }
  /* rn: the FP64 residual the sweep started from; returns 1 when the solve
   * must stop */
  int after_sweep(int inner_iters, double rn, const char *what)
  {
    used += inner_iters;
    int stop = 0;
    if(sweeps >= 2 && hist[0] >= 0. && !(rn <= 0.5 * hist[0])) {
      if(g_opt.verbose)
        fprintf(stderr, "%s: FP64 residual %.3e not below half of %.3e two "
          "sweeps earlier: stopping\n", what, rn, hist[0]);
      stop = 1;
    }
    if(remaining() <= 0) {
      if(g_opt.verbose)
        fprintf(stderr, "%s: inner iteration budget %d spent\n", what, budget);
      stop = 1;
    }
    hist[0] = hist[1];
    hist[1] = rn;
    sweeps++;
    return stop;
  }
};

/* runs after k_pp_rhs has filled b, x and s->bnorm */
template <int VD, int VF>
static int poisson_mixed(const boxc &BD, const boxc &BF, const opc &O,
  long long n, int record)
{
  ensure_fp32();
  bbb_kry *s = g_dev.kry, *si = g_dev.kry_inner;
  dim3 grdD = box_grid(BD), blk(TX, TY);
  bbb_kry init;
  memset(&init, 0, sizeof(init));
  BBB_CK(cudaMemcpyAsync(g_dev.kry_host, s, sizeof(bbb_kry),
    cudaMemcpyDeviceToHost, g_dev.stream));
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
  init.bnorm = g_dev.kry_host->bnorm;
  init.tol = bbb_pp_tol() * init.bnorm;
  init.maxit = g_opt.max_outer > 0 ? g_opt.max_outer : 40;
  BBB_CK(cudaMemcpyAsync(s, &init, sizeof(bbb_kry), cudaMemcpyHostToDevice,
    g_dev.stream));
  int project = (nparts == 0) && (bc.pW == bc.pE) && (bc.pS == bc.pN)
    && (bc.pB == bc.pT);
  double itol = g_opt.inner_tol > 0 ? g_opt.inner_tol : 1e-4;
  int inner_total = 0, cur = 0, fresh = 1, resume_failed = 0;
  dc_guard guard(pp_max_iter);
  for(int outer = 0; outer <= init.maxit; outer++) {
    outer_resid<VD>(BD, O, g_dev.mask_p, g_dev.kb, g_dev.kx, g_dev.fb, s, si,
      itol, guard.remaining(), project, n);
    /* a sweep starts the FP32 BiCGSTAB from e = 0; with reliable updates
     * later sweeps replace its residual by the FP64 one and carry on
     * (restarting only after an inner breakdown).  On the 256x256x512
     * sedimentation box both take about the FP64 form's iteration count
     * (restarts at 1e-4: ~500 per step; reliable at 1e-2: ~480 with twice
     * the sweeps), so restarting is the default. */
    if(fresh) {
      k_inner_setup<VF><<<NPW, 256, 0, g_dev.stream>>>(n, g_dev.fb, g_dev.fs,
        g_dev.fx, g_dev.frh, si, g_dev.partials);
      cur = 0;
    } else {
      k_reliable_setup<VF><<<NPW, 256, 0, g_dev.stream>>>(n, g_dev.fb, g_dev.frh,
        g_dev.fr, g_dev.fx, si, g_dev.partials);
    }
    BBB_LAUNCHED();
    bicgstab_iterations<float, VF>(BF, O, n, g_dev.mask_p, g_dev.fr, g_dev.frh,
      g_dev.fp[0], g_dev.fp[1], g_dev.fv[0], g_dev.fv[1], g_dev.fs, g_dev.ft,
      g_dev.fx, si, guard.remaining(), 4, &cur, !fresh);
    if(bbb_last_status() == BBB_ERR_CUDA) return -1;
    inner_total += g_dev.kry_host->iter;
    if(g_opt.verbose)
      fprintf(stderr, "poisson mixed sweep %d (%s): %d inner iterations, "
        "converged %d, s_conv %d, status %d, ||r_inner|| %.3e (tol %.3e)\n",
        outer, fresh ? "fresh" : "resumed", g_dev.kry_host->iter,
        g_dev.kry_host->converged, g_dev.kry_host->s_conv,
        g_dev.kry_host->status, g_dev.kry_host->rnorm, g_dev.kry_host->tol);
    /* a breakdown (non-finite scalar, or a resumed sweep whose residual
     * grew 1e3-fold: the shadow residual no longer correlates with the
     * replaced one) or a sweep that ran out of iterations: the next sweep
     * restarts from the FP64 residual, and after a failed resumption the
     * rest of this solve restarts every sweep */
    int broke = g_dev.kry_host->status != 0;
    if(broke) {
      /* the FP64 solution is untouched by a failed sweep's e */
      cudaMemsetAsync(g_dev.fx, 0, sizeof(float) * (size_t)n, g_dev.stream);
      if(!fresh) resume_failed = 1;
    }
    fresh = !g_opt.reliable || broke || resume_failed
      || !g_dev.kry_host->converged || g_dev.kry_host->s_conv;
    k_accumulate<VF><<<NPW, 256, 0, g_dev.stream>>>(n, g_dev.kx, g_dev.fx, s);
    BBB_LAUNCHED();
    BBB_CK(cudaMemcpyAsync(g_dev.kry_host, s, sizeof(bbb_kry),
      cudaMemcpyDeviceToHost, g_dev.stream));
    BBB_CK(cudaStreamSynchronize(g_dev.stream));
    if(g_opt.verbose)
      fprintf(stderr, "poisson mixed sweep %d: FP64 ||r|| %.3e (tol %.3e)\n",
        outer, g_dev.kry_host->rnorm, g_dev.kry_host->tol);
    if(g_dev.kry_host->done) break;
    if(guard.after_sweep(inner_total - guard.used, g_dev.kry_host->rnorm,
                         "pressure-Poisson (mixed)"))
      break;
  }
  bbb_kry *h = g_dev.kry_host;
  real resid = h->bnorm > 0 ? h->rnorm / h->bnorm : h->rnorm;
  if(g_stats.pp_solves == 0) g_stats.pp_iters_first = inner_total;
  g_stats.pp_solves++;
  g_stats.pp_iters_total += inner_total;
  g_stats.pp_iters_last = inner_total;
  if(inner_total > g_stats.pp_iters_max) g_stats.pp_iters_max = inner_total;
  g_stats.pp_resid_last = resid;
  g_stats.pp_outer_last = h->iter;
  if(record) bbb_record_solver("solver_expd.rec", inner_total, resid);
  return h->converged ? inner_total : -inner_total;
}

int bbb_poisson_solve_mixed(int record)
{
  bbb_dev_require();
  if(!g_dev.ready) return -1;
  bbb_build_masks();
  bbb_geom G = bbb_make_geom();
  int VD = pick_vec(G.nx, sizeof(double)), VF = pick_vec(G.nx, sizeof(float));
  int px = bc.pW == BBB_PERIODIC, py = bc.pS == BBB_PERIODIC, pz = bc.pB == BBB_PERIODIC;
  int smD = resident(k_outer_resid<1>);
  if(VD == 2) smD = resident(k_outer_resid<2>);
  int smF = VF == 4 ? bicg_per_sm<float, 4>() : bicg_per_sm<float, 1>();
  boxc BD = make_box(G.nx, G.ny, G.nz, px, py, pz, 0, 0, 0, VD, smD);
  boxc BF = make_box(G.nx, G.ny, G.nz, px, py, pz, 0, 0, 0, VF, smF);
  opc O = poisson_op(G);
  long long n = (long long)G.nx * G.ny * G.nz;
  k_pp_rhs<<<NPW, 256, 0, g_dev.stream>>>(g_dev.us, g_dev.vs, g_dev.ws,
    g_dev.phi, g_dev.phase, G, rho_f / dt, g_dev.kb, g_dev.kx, g_dev.kry,
    g_dev.partials);
  BBB_LAUNCHED();
  bbb_learn_pre_solve();
  int it;
  if(VD == 2 && VF == 4) it = poisson_mixed<2, 4>(BD, BF, O, n, record);
  else if(VD == 2 && VF == 1) it = poisson_mixed<2, 1>(BD, BF, O, n, record);
  else it = poisson_mixed<1, 1>(BD, BF, O, n, record);
  k_pp_writeback<<<NPW, 256, 0, g_dev.stream>>>(g_dev.kx, g_dev.phi, G, g_dev.kry);
  BBB_LAUNCHED();
  bbb_learn_post_solve();
  bbb_kry *h = g_dev.kry_host;
  bbb_learn_solve_done(h->rnorm);
  if(h->status == BBB_ERR_NONFINITE) bbb_set_status(BBB_ERR_NONFINITE, "pressure-Poisson");
  if(!h->converged) {
    bbb_set_status(BBB_ERR_NOT_CONVERGED, "pressure-Poisson (mixed)");
    if(bbb_fail_exit()) {
      printf("The pressure-Poisson equation did not converge.              \n");
      exit(EXIT_FAILURE);
    }
  }
  return it;
}

/* ||b - A x|| of the pressure system for an FP64 candidate x (dense), on
 * the current b (kb) and operator mask: the gate of the learned guess */
struct epi_rn {
  const double *b;
  template <int V>
  __device__ __forceinline__ void at(long long c, const double (&xr)[V],
    const double (&Ax)[V], double (&red)[1]) const
  {
    double bb[V];
    ldv<double, V>(b, c, bb);
#pragma unroll
    for(int a = 0; a < V; a++) { double r = bb[a] - Ax[a]; red[0] += r * r; }
    (void)xr;
  }
};

template <int V>
__global__ void __launch_bounds__(NTHR) k_resid_norm(boxc B, opc O,
  const uint8_t *__restrict__ mask, const double *__restrict__ b,
  const double *x, double *partials, unsigned int *ticket, double *out)
{
  __shared__ double sh[32];
  __shared__ optab<double> tab;
  optab_fill<double>(tab, O);
  prod_x<double> P{x};
  epi_rn E{b};
  double red[1] = {0.};
  tile_stencil<double, V>(B, O, mask, tab, P, E, red);
  if(bbb_grid_partial<1>(red, partials, ticket, sh)) {
    bbb_grid_finish_sum<1>(red, partials, ticket, sh);
    if(threadIdx.x == 0 && threadIdx.y == 0) *out = sqrt(red[0]);
  }
}

double bbb_poisson_resid_norm(const double *x)
{
  bbb_build_masks();
  bbb_geom G = bbb_make_geom();
  int V = pick_vec(G.nx, sizeof(double));
  static int sm1 = 0, sm2 = 0;
  if(!sm1) { sm1 = resident(k_resid_norm<1>); sm2 = resident(k_resid_norm<2>); }
  boxc B = make_box(G.nx, G.ny, G.nz, bc.pW == BBB_PERIODIC,
    bc.pS == BBB_PERIODIC, bc.pB == BBB_PERIODIC, 0, 0, 0, V, V == 2 ? sm2 : sm1);
  opc O = poisson_op(G);
  dim3 grd = box_grid(B), blk(TX, TY);
  if(V == 2)
    k_resid_norm<2><<<grd, blk, 0, g_dev.stream>>>(B, O, g_dev.mask_p, g_dev.kb,
      x, g_dev.partials, g_dev.red_ticket + 10, g_dev.red_dev + 48);
  else
    k_resid_norm<1><<<grd, blk, 0, g_dev.stream>>>(B, O, g_dev.mask_p, g_dev.kb,
      x, g_dev.partials, g_dev.red_ticket + 10, g_dev.red_dev + 48);
  BBB_LAUNCHED();
  double r = -1.;
  BBB_CK(cudaMemcpyAsync(g_dev.red_host, g_dev.red_dev + 48, sizeof(double),
    cudaMemcpyDeviceToHost, g_dev.stream));
  BBB_CK(cudaStreamSynchronize(g_dev.stream));
  r = g_dev.red_host[0];
  return r;
}

/* src/cuda_bicgstab.cu:715-1073 */
extern "C" void cuda_PP_bicgstab(int rank)
{
  (void)rank;
  if(g_opt.precision == BBB_PREC_MIXED) bbb_poisson_solve_mixed(1);
  else bbb_poisson_solve(1);
}

/* src/cuda_bicgstab.cu:1178-1204: the un-ghosted Poisson right-hand side
 * (kept for callers that use it on its own) */
extern "C" void cuda_PP_rhs(int dev)
{
  (void)dev;
  bbb_dev_require();
  if(!g_dev.ready) return;
  bbb_geom G = bbb_make_geom();
  k_pp_rhs<<<NPW, 256, 0, g_dev.stream>>>(g_dev.us, g_dev.vs, g_dev.ws,
    g_dev.phi, g_dev.phase, G, rho_f / dt, g_dev.kb, g_dev.kx, g_dev.kry,
    g_dev.partials);
  BBB_LAUNCHED();
}

/* ------------------------------------------------ Helmholtz CG */

template <typename T>
struct prod_c1 {
  const T *r, *p; const uint8_t *mask; T beta; int first;
  typedef T Raw;
  template <int V>
  __device__ __forceinline__ void ev(long long c, T (&raw)[V], T (&q)[V],
    const T *dinv, bool own, double (&red)[1]) const
  {
    T pp[V];
    ldv<T, V>(p, c, pp);
    if(first) {
#pragma unroll
      for(int a = 0; a < V; a++) raw[a] = pp[a];
    } else {
      T rr[V];
      unsigned mm[V];
      ldv<T, V>(r, c, rr);
      ldm<V>(mask, c, mm);
#pragma unroll
      for(int a = 0; a < V; a++) raw[a] = (T)1. * (dinv[mm[a]] * rr[a]) + beta * pp[a];
    }
#pragma unroll
    for(int a = 0; a < V; a++) q[a] = raw[a];
    (void)own; (void)red;
  }
};
template <typename T>
struct epi_c1 {
  T *pn, *y;
  template <int V>
  __device__ __forceinline__ void at(long long c, const T (&praw)[V],
    const T (&Ap)[V], double (&red)[1]) const
  {
    stv<T, V>(pn, c, praw);
    stv<T, V>(y, c, Ap);
#pragma unroll
    for(int a = 0; a < V; a++) red[0] += (double)Ap[a] * (double)praw[a];
  }
};

template <typename T, int V>
__global__ void __launch_bounds__(NTHR) k_cg1(boxc B, opc O,
  const uint8_t *__restrict__ mask, const T *r, const T *p_old, T *p_new,
  T *y, bbb_kry *s, double *partials)
{
  if(((volatile bbb_kry *)s)->done) return;
  __shared__ double sh[32];
  __shared__ optab<T> tab;
  optab_fill<T>(tab, O);
  prod_c1<T> P{r, p_old, mask, (T)s->beta, s->first};
  epi_c1<T> E{p_new, y};
  double red[1] = {0.};
  tile_stencil<T, V>(B, O, mask, tab, P, E, red);
  if(bbb_grid_partial<1>(red, partials, &s->ticket, sh)) {
    bbb_grid_finish_sum<1>(red, partials, &s->ticket, sh);
    if(threadIdx.x == 0 && threadIdx.y == 0) {
      s->alpha = s->rho / red[0];
      s->first = 0;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_cg2(long long n, opc O,
  const uint8_t *__restrict__ mask, T *x, const T *__restrict__ p, T *r,
  const T *__restrict__ y, bbb_kry *s, double *partials)
{
  if(((volatile bbb_kry *)s)->done) return;
  __shared__ double sh[32 * 2];
  __shared__ optab<T> tab;
  optab_fill<T>(tab, O);
  T a = (T)s->alpha;
  double red[2] = {0., 0.};
  /* 16 bytes per array and thread per step (the vectors start 256-byte
   * aligned); the n % V cells past the last full vector by the first
   * threads */
  constexpr int V = 16 / (int)sizeof(T);
  const long long nv = n / V;
  const long long tid0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for(long long q = tid0; q < nv; q += stride) {
    const long long c = q * V;
    T pv[V], xv[V], yv[V], rv[V];
    ldv<T, V>(p, c, pv); ldv<T, V>(x, c, xv);
    ldv<T, V>(y, c, yv); ldv<T, V>(r, c, rv);
    unsigned mw;
    if constexpr(V == 4) mw = *reinterpret_cast<const unsigned *>(mask + c);
    else mw = *reinterpret_cast<const unsigned short *>(mask + c);
#pragma unroll
    for(int v = 0; v < V; v++) {
      xv[v] = a * pv[v] + xv[v];
      rv[v] = -a * yv[v] + rv[v];
      T z = tab.dinv[(mw >> (8 * v)) & 0xffu] * rv[v];
      red[0] += (double)rv[v] * (double)z;
      red[1] += (double)rv[v] * (double)rv[v];
    }
    stv<T, V>(x, c, xv); stv<T, V>(r, c, rv);
  }
  for(long long c = nv * V + tid0; c < n; c += stride) {
    T pv = p[c];
    x[c] = a * pv + x[c];
    T rv = -a * y[c] + r[c];
    r[c] = rv;
    T z = tab.dinv[mask[c]] * rv;
    red[0] += (double)rv * (double)z;
    red[1] += (double)rv * (double)rv;
  }
  if(bbb_grid_partial<2>(red, partials, &s->ticket, sh)) {
    bbb_grid_finish_sum<2>(red, partials, &s->ticket, sh);
    if(threadIdx.x == 0) {
      s->beta = red[0] / s->rho;
      s->rho = red[0];
      s->iter += 1;
      double rn = sqrt(red[1]);
      s->rnorm = rn;
      s->converged = (rn <= s->tol);
      if(!isfinite(rn)) { s->status = BBB_ERR_NONFINITE; s->done = 1; }
      if(s->converged || s->iter >= s->maxit) s->done = 1;
    }
  }
}

/* b = u* on the interior faces of the component, x = 0, r = b, p = M r */
__global__ void k_cg_setup(const real *star, bbb_geom G, int comp, int nx,
  int ny, int nz, int tr, opc O, const uint8_t *mask, double *x, double *r,
  double *p, bbb_kry *s, double *partials, double rtol, int maxit)
{
  __shared__ double sh[32 * 2];
  __shared__ optab<double> tab;
  optab_fill<double>(tab, O);
  int s1 = comp == 0 ? G.fx_s1 : (comp == 1 ? G.fy_s1 : G.fz_s1);
  int s2 = comp == 0 ? G.fx_s2 : (comp == 1 ? G.fy_s2 : G.fz_s2);
  long long n = (long long)nx * ny * nz;
  double red[2] = {0., 0.};
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    helm_ijk(t, nx, ny, tr, i, j, k);
    double bv = star[i + (long long)j * s1 + (long long)k * s2];
    x[t] = 0.;
    r[t] = bv;
    double z = tab.dinv[mask[t]] * bv;
    p[t] = z;
    red[0] += bv * z;
    red[1] += bv * bv;
  }
  if(bbb_grid_partial<2>(red, partials, &s->ticket, sh)) {
    bbb_grid_finish_sum<2>(red, partials, &s->ticket, sh);
    if(threadIdx.x == 0) {
      double rn = sqrt(red[1]);
      s->rho = red[0];
      s->bnorm = rn;
      s->rnorm = rn;
      s->tol = rtol * rn;
      s->iter = 0;
      s->maxit = maxit;
      s->first = 1;
      s->beta = 0.;
      s->converged = (rn <= s->tol);
      s->done = s->converged || (maxit <= 0) || !isfinite(rn);
      s->status = isfinite(rn) ? 0 : BBB_ERR_NONFINITE;
    }
  }
}

__global__ void k_cg_writeback(const double *x, real *star, bbb_geom G,
  int comp, int nx, int ny, int nz, int tr)
{
  int s1 = comp == 0 ? G.fx_s1 : (comp == 1 ? G.fy_s1 : G.fz_s1);
  int s2 = comp == 0 ? G.fx_s2 : (comp == 1 ? G.fy_s2 : G.fz_s2);
  long long n = (long long)nx * ny * nz;
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    helm_ijk(t, nx, ny, tr, i, j, k);
    star[i + (long long)j * s1 + (long long)k * s2] = x[t];
  }
}

/* The Crank-Nicolson system of velocity component `comp`: its box (the
 * component's faces, x-fastest, or for the u system y-fastest where
 * helm_tr says so), periodic and duplicated-face flags per box axis, and
 * the operator weights 0.5 nu dt / h^2 along the box axes. */
struct helm_box {
  int nx, ny, nz, px, py, pz, dx, dy, dz, tr;
  opc O;
};

static helm_box helm_system(int comp, const bbb_geom &G)
{
  helm_box h;
  int per[3][3] = {{bc.uW, bc.uS, bc.uB}, {bc.vW, bc.vS, bc.vB}, {bc.wW, bc.wS, bc.wB}};
  int fx = G.nx + (comp == 0), fy = G.ny + (comp == 1), fz = G.nz + (comp == 2);
  int px = per[comp][0] == BBB_PERIODIC, py = per[comp][1] == BBB_PERIODIC;
  double wx = 0.5 * nu * dt * (1. / (G.dx * G.dx));
  double wy = 0.5 * nu * dt * (1. / (G.dy * G.dy));
  h.tr = helm_tr(comp, G);
  h.nx = h.tr ? fy : fx; h.ny = h.tr ? fx : fy; h.nz = fz;
  h.px = h.tr ? py : px; h.py = h.tr ? px : py;
  h.pz = per[comp][2] == BBB_PERIODIC;
  h.dx = h.tr ? comp == 1 : comp == 0;
  h.dy = h.tr ? comp == 0 : comp == 1;
  h.dz = comp == 2;
  h.O.wx = h.tr ? wy : wx;
  h.O.wy = h.tr ? wx : wy;
  h.O.wz = 0.5 * nu * dt * (1. / (G.dz * G.dz));
  h.O.helm = 1;
  return h;
}

/* ------------------------------------------------ mixed-precision CG
 * The Crank-Nicolson Helmholtz solves in the FP32-inner form: FP64 outer
 * residual r = b - A x (b = u* on the component's faces, x from 0), FP32
 * Jacobi-CG on A e = r to `inner_tol` (or looser when half the remaining
 * reduction suffices), x += e in FP64; stops on the FP64 test
 * ||r|| <= pp_residual ||b|| of the FP64 form. */

/* b = u* (dense FP64), x = 0, ||b||; the finaliser sets up the outer
 * scalars */
__global__ void k_helm_b(const real *star, bbb_geom G, int comp, int nx,
  int ny, int nz, int tr, double *b, double *x, bbb_kry *s, double *partials,
  double rtol, int max_outer)
{
  __shared__ double sh[32];
  int s1 = comp == 0 ? G.fx_s1 : (comp == 1 ? G.fy_s1 : G.fz_s1);
  int s2 = comp == 0 ? G.fx_s2 : (comp == 1 ? G.fy_s2 : G.fz_s2);
  long long n = (long long)nx * ny * nz;
  double red[1] = {0.};
  for(long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
      t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    helm_ijk(t, nx, ny, tr, i, j, k);
    double bv = star[i + (long long)j * s1 + (long long)k * s2];
    b[t] = bv;
    x[t] = 0.;
    red[0] += bv * bv;
  }
  if(bbb_grid_partial<1>(red, partials, &s->ticket, sh)) {
    bbb_grid_finish_sum<1>(red, partials, &s->ticket, sh);
    if(threadIdx.x == 0) {
      double bn = sqrt(red[0]);
      s->bnorm = bn;
      s->rnorm = bn;
      s->tol = rtol * bn;
      s->iter = 0;
      s->maxit = max_outer;
      s->converged = 0;
      s->done = 0;
      s->status = isfinite(bn) ? 0 : BBB_ERR_NONFINITE;
      if(!isfinite(bn)) s->done = 1;
    }
  }
}

/* FP32 inner CG from e = 0: z = M r, p = z, (r, z), ||r|| */
template <int V>
__global__ void __launch_bounds__(256) k_cg_inner_setup(long long n, opc O,
  const uint8_t *__restrict__ mask, const float *__restrict__ r, float *e,
  float *p, bbb_kry *si, double *partials)
{
  if(((volatile bbb_kry *)si)->done) return;
  __shared__ double sh[32 * 2];
  __shared__ optab<float> tab;
  optab_fill<float>(tab, O);
  double red[2] = {0., 0.};
  long long nv = n / V;
  for(long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nv;
      q += (long long)gridDim.x * blockDim.x) {
    long long c = q * V;
    float rv[V], z[V], zero[V];
    unsigned mm[V];
    ldv<float, V>(r, c, rv);
    ldm<V>(mask, c, mm);
#pragma unroll
    for(int a = 0; a < V; a++) {
      z[a] = tab.dinv[mm[a]] * rv[a];
      zero[a] = 0.f;
      red[0] += (double)rv[a] * (double)z[a];
      red[1] += (double)rv[a] * (double)rv[a];
    }
    stv<float, V>(p, c, z);
    stv<float, V>(e, c, zero);
  }
  if(bbb_grid_partial<2>(red, partials, &si->ticket, sh)) {
    bbb_grid_finish_sum<2>(red, partials, &si->ticket, sh);
    if(threadIdx.x == 0) {
      double rn = sqrt(red[1]);
      si->rho = red[0];
      si->rnorm = rn;
      si->iter = 0;
      si->first = 1;
      si->beta = 0.;
      si->converged = (rn <= si->tol);
      si->done = si->converged || si->maxit <= 0 || !isfinite(rn);
      si->status = isfinite(rn) ? 0 : BBB_ERR_NONFINITE;
    }
  }
}

/* The Helmholtz CG stencil pass (p = M r + beta p_old, y = A p, (p, y))
 * staged by tensor-map copies where the rows are a multiple of 128 cells
 * (the v and w systems of a 256-wide box; the u system carries the
 * duplicated periodic face and stays on the register-tiled k_cg1).  Maps
 * for both direction buffers are made once per solve. */
template <typename T>
struct cg_staged {
  bool on = false;
  boxc B;
  as_maps M[2];
  cg_staged(const boxc &B0, const uint8_t *mask, const T *r, T *const *p)
  {
    B = B0;
    on = BBB_ASYNC_ON && B0.nx % AS_W == 0 && as_per_sm<T, 3>() > 0;
    if(!on) return;
    B = retile(B0, as_per_sm<T, 3>(), as_layout<T, 3>::ALIGN, as_layout<T, 3>::TH);
    for(int c = 0; c < 2 && on; c++) {
      const T *h[4] = {r, p[c], NULL, NULL};
      on = as_pass_maps<T, 3>(&M[c], B, mask, h, NULL);
    }
  }
  /* reads r and p[cur], writes p[cur ^ 1] and y */
  void launch(const opc &O, const uint8_t *mask, const T *r, T *const *p,
    int cur, T *y, bbb_kry *s) const
  {
    as_args<T> A = {};
    A.mask = mask;
    A.h[0] = r; A.h[1] = p[cur];
    A.w0 = p[cur ^ 1]; A.w1 = y;
    A.s = s; A.partials = g_dev.partials;
    k_bicg_async<T, 3><<<B.nblk, as_layout<T, 3>::THREADS, as_layout<T, 3>::SMEM,
      g_dev.stream>>>(B, O, A, M[cur]);
  }
};

template <int VD, int VF>
static int helmholtz_mixed(const boxc &BD, const boxc &BF, const opc &O,
  const uint8_t *mask, long long n, bbb_geom G, int comp, int tr, real *star)
{
  ensure_fp32();
  bbb_kry *s = g_dev.kry, *si = g_dev.kry_inner;
  int max_outer = g_opt.max_outer > 0 ? g_opt.max_outer : 20;
  double itol = g_opt.inner_tol > 0 ? g_opt.inner_tol : 1e-4;
  int nx = BD.nx, ny = BD.ny, nz = BD.nz;
  k_helm_b<<<NPW, 256, 0, g_dev.stream>>>(star, G, comp, nx, ny, nz, tr, g_dev.kb,
    g_dev.kx, s, g_dev.partials, pp_residual, max_outer);
  BBB_LAUNCHED();
  dim3 grdD = box_grid(BD), grdF = box_grid(BF), blk(TX, TY);
  int inner_total = 0;
  dc_guard guard(pp_max_iter);
  const cg_staged<float> CS(BF, mask, g_dev.fr, g_dev.fp);
  for(int outer = 0; outer <= max_outer; outer++) {
    outer_resid<VD>(BD, O, mask, g_dev.kb, g_dev.kx, g_dev.fr, s, si, itol,
      guard.remaining(), 0, n);
    k_cg_inner_setup<VF><<<NPW, 256, 0, g_dev.stream>>>(n, O, mask, g_dev.fr,
      g_dev.fx, g_dev.fp[0], si, g_dev.partials);
    BBB_LAUNCHED();
    int cur = 0;
    const int pmark = prof_mark();
    drive(si, [&]() {
      prof_begin(BBB_PROF_CG1, (double)n * (4. * 4. + 1.));
      if(CS.on)
        CS.launch(O, mask, g_dev.fr, g_dev.fp, cur, g_dev.fv[0], si);
      else
        k_cg1<float, VF><<<grdF, blk, 0, g_dev.stream>>>(BF, O, mask, g_dev.fr,
          g_dev.fp[cur], g_dev.fp[cur ^ 1], g_dev.fv[0], si, g_dev.partials);
      BBB_LAUNCHED();
      prof_end();
      prof_begin(BBB_PROF_CG2, (double)n * (6. * 4. + 1.));
      k_cg2<float><<<NPW, 256, 0, g_dev.stream>>>(n, O, mask, g_dev.fx,
        g_dev.fp[cur ^ 1], g_dev.fr, g_dev.fv[0], si, g_dev.partials);
      BBB_LAUNCHED();
      prof_end();
      cur ^= 1;
    }, guard.remaining(), 2);
    if(bbb_last_status() == BBB_ERR_CUDA) return -1;
    prof_ran(pmark, 2LL * g_dev.kry_host->iter);
    prof_collect();
    inner_total += g_dev.kry_host->iter;
    k_accumulate<VF><<<NPW, 256, 0, g_dev.stream>>>(n, g_dev.kx, g_dev.fx, s);
    BBB_LAUNCHED();
    BBB_CK(cudaMemcpyAsync(g_dev.kry_host, s, sizeof(bbb_kry),
      cudaMemcpyDeviceToHost, g_dev.stream));
    BBB_CK(cudaStreamSynchronize(g_dev.stream));
    if(g_dev.kry_host->done) break;
    if(guard.after_sweep(inner_total - guard.used, g_dev.kry_host->rnorm,
                         "Helmholtz (mixed)"))
      break;
  }
  k_cg_writeback<<<NPW, 256, 0, g_dev.stream>>>(g_dev.kx, star, G, comp,
    nx, ny, nz, tr);
  BBB_LAUNCHED();
  return inner_total;
}

int bbb_helmholtz_solve(int comp)
{
  bbb_dev_require();
  if(!g_dev.ready) return -1;
  if(g_opt.precision == BBB_PREC_MIXED) {
    bbb_build_masks();
    bbb_geom G = bbb_make_geom();
    helm_box hb = helm_system(comp, G);
    int nx = hb.nx, ny = hb.ny, nz = hb.nz, tr = hb.tr;
    int px = hb.px, py = hb.py, pz = hb.pz;
    int VD = pick_vec(nx, sizeof(double)), VF = pick_vec(nx, sizeof(float));
    static int smd[3], smf[3];
    if(!smd[0]) {
      smd[1] = resident(k_outer_resid<1>); smd[2] = resident(k_outer_resid<2>);
      smf[1] = resident(k_cg1<float, 1>); smf[2] = resident(k_cg1<float, 4>);
      smd[0] = 1;
    }
    boxc BD = make_box(nx, ny, nz, px, py, pz, hb.dx, hb.dy, hb.dz,
      VD, smd[VD == 2 ? 2 : 1]);
    boxc BF = make_box(nx, ny, nz, px, py, pz, hb.dx, hb.dy, hb.dz,
      VF, smf[VF == 4 ? 2 : 1]);
    opc O = hb.O;
    const uint8_t *mask = comp == 0 ? g_dev.mask_u : (comp == 1 ? g_dev.mask_v : g_dev.mask_w);
    real *star = comp == 0 ? g_dev.us : (comp == 1 ? g_dev.vs : g_dev.ws);
    long long n = (long long)nx * ny * nz;
    int it;
    if(VD == 2 && VF == 4) it = helmholtz_mixed<2, 4>(BD, BF, O, mask, n, G, comp, tr, star);
    else if(VD == 2) it = helmholtz_mixed<2, 1>(BD, BF, O, mask, n, G, comp, tr, star);
    else it = helmholtz_mixed<1, 1>(BD, BF, O, mask, n, G, comp, tr, star);
    bbb_kry *h = g_dev.kry_host;
    real resid = h->bnorm > 0 ? h->rnorm / h->bnorm : h->rnorm;
    g_stats.helm_iters_total += it > 0 ? it : 0;
    g_stats.helm_solves++;
    bbb_record_solver("solver_helmholtz_expd.rec", it, resid);
    if(h->status == BBB_ERR_NONFINITE) bbb_set_status(BBB_ERR_NONFINITE, "Helmholtz");
    if(!h->converged) {
      bbb_set_status(BBB_ERR_NOT_CONVERGED, "Helmholtz (mixed)");
      if(bbb_fail_exit()) {
        printf("The Helmholtz equation did not converge.              \n");
        exit(EXIT_FAILURE);
      }
    }
    return it;
  }
  bbb_build_masks();
  bbb_geom G = bbb_make_geom();
  helm_box hb = helm_system(comp, G);
  int nx = hb.nx, ny = hb.ny, nz = hb.nz, tr = hb.tr;
  int V = pick_vec(nx, sizeof(double));
  static int sm1 = 0, sm2 = 0;
  if(!sm1) { sm1 = resident(k_cg1<double, 1>); sm2 = resident(k_cg1<double, 2>); }
  boxc B = make_box(nx, ny, nz, hb.px, hb.py, hb.pz, hb.dx, hb.dy, hb.dz, V,
    V == 2 ? sm2 : sm1);
  opc O = hb.O;
  const uint8_t *mask = comp == 0 ? g_dev.mask_u : (comp == 1 ? g_dev.mask_v : g_dev.mask_w);
  real *star = comp == 0 ? g_dev.us : (comp == 1 ? g_dev.vs : g_dev.ws);
  long long n = (long long)nx * ny * nz;
  bbb_kry *s = g_dev.kry;
  k_cg_setup<<<NPW, 256, 0, g_dev.stream>>>(star, G, comp, nx, ny, nz, tr, O,
    mask, g_dev.kx, g_dev.kr, g_dev.kp[0], s, g_dev.partials, pp_residual,
    pp_max_iter);
  BBB_LAUNCHED();
  dim3 grd = box_grid(B), blk(TX, TY);
  int cur = 0;
  const int pmark = prof_mark();
  const cg_staged<double> CS(B, mask, g_dev.kr, g_dev.kp);
  drive(s, [&]() {
    prof_begin(BBB_PROF_CG1, (double)n * (4. * 8. + 1.));
    if(CS.on)
      CS.launch(O, mask, g_dev.kr, g_dev.kp, cur, g_dev.kv[0], s);
    else if(V == 2)
      k_cg1<double, 2><<<grd, blk, 0, g_dev.stream>>>(B, O, mask, g_dev.kr,
        g_dev.kp[cur], g_dev.kp[cur ^ 1], g_dev.kv[0], s, g_dev.partials);
    else
      k_cg1<double, 1><<<grd, blk, 0, g_dev.stream>>>(B, O, mask, g_dev.kr,
        g_dev.kp[cur], g_dev.kp[cur ^ 1], g_dev.kv[0], s, g_dev.partials);
    BBB_LAUNCHED();
    prof_end();
    prof_begin(BBB_PROF_CG2, (double)n * (6. * 8. + 1.));
    k_cg2<double><<<NPW, 256, 0, g_dev.stream>>>(n, O, mask, g_dev.kx,
      g_dev.kp[cur ^ 1], g_dev.kr, g_dev.kv[0], s, g_dev.partials);
    BBB_LAUNCHED();
    prof_end();
    cur ^= 1;
  }, pp_max_iter, 1);
  prof_ran(pmark, 2LL * g_dev.kry_host->iter);
  prof_collect();
  k_cg_writeback<<<NPW, 256, 0, g_dev.stream>>>(g_dev.kx, star, G, comp,
    nx, ny, nz, tr);
  BBB_LAUNCHED();
  bbb_kry *h = g_dev.kry_host;
  real resid = h->bnorm > 0 ? h->rnorm / h->bnorm : h->rnorm;
  g_stats.helm_iters_total += h->iter;
  g_stats.helm_solves++;
  bbb_record_solver("solver_helmholtz_expd.rec", h->iter, resid);
  if(h->status == BBB_ERR_NONFINITE) bbb_set_status(BBB_ERR_NONFINITE, "Helmholtz");
  if(!h->converged) {
    bbb_set_status(BBB_ERR_NOT_CONVERGED, "Helmholtz");
    if(bbb_fail_exit()) {
      printf("The Helmholtz equation did not converge.              \n");
      exit(EXIT_FAILURE);
    }
  }
  return h->iter;
}

/* src/cuda_bicgstab.cu:44-316 (and the v, w variants): RHS, boundary
 * conditions on u*, particle velocities on u*, then the CG solve */
static void helmholtz_entry(int comp)
{
  bbb_star_rhs(1 << comp, 0);
  cuda_dom_BC_star();
  if(nparts > 0) cuda_part_BC_star();
  bbb_helmholtz_solve(comp);
}

extern "C" void cuda_ustar_helmholtz(int rank) { (void)rank; helmholtz_entry(0); }
extern "C" void cuda_vstar_helmholtz(int rank) { (void)rank; helmholtz_entry(1); }
extern "C" void cuda_wstar_helmholtz(int rank) { (void)rank; helmholtz_entry(2); }

/* ------------------------------------------------ allocation-free solve
 * bbb_PP_bicgstab_static: the FP64 pressure-Poisson solve of
 * cuda_PP_bicgstab for callers that cannot allocate device memory -- for
 * example a host application whose own pool allocator owns all of the
 * GPU's memory, or a time-critical loop that cannot afford the implicit
 * device synchronisation cudaMalloc/cudaFree bring.  The caller passes the
 * inputs and the output as device pointers; everything else (operator
 * mask, Krylov vectors, reduction partials, solver scalars) lives in the
 * fixed array below, which every GPU that loads this library holds until
 * the process exits.  No cudaMalloc, cudaFree or allocating library call
 * is made. */
#define BBB_STATIC_MAX_CELLS (64LL * 64LL * 64LL)
#define BBB_STATIC_PARTIALS (16384LL * 5LL)
#define BBB_STATIC_SCRATCH_BYTES \
  (256LL + 256LL * ((BBB_STATIC_PARTIALS * 8LL + 255LL) / 256LL) \
   + 256LL * ((BBB_STATIC_MAX_CELLS + 255LL) / 256LL) \
   + 10LL * 256LL * ((BBB_STATIC_MAX_CELLS * 8LL + 255LL) / 256LL))

static __device__ __align__(256) unsigned char
  g_static_scratch[BBB_STATIC_SCRATCH_BYTES];

/* device address of g_static_scratch per device, looked up once with that
 * device current; the lock makes host threads that make their first call
 * on a device at the same time take one look-up */
static unsigned char *g_static_addr[64];
static std::mutex g_static_lock;

template <int V>
static int static_iterations(const boxc &B, const opc &O, const uint8_t *mask,
  double *b, double *x, double *r, double *rh, double *const *pp,
  double *const *vv, double *sv, double *tv, bbb_kry *s, double *partials,
  double tol, int maxit, cudaStream_t st, bbb_kry *h)
{
  dim3 grd = box_grid(B), blk(TX, TY);
  k_bicg_setup<double, V><<<grd, blk, 0, st>>>(B, O, mask, b, x, sv, rh, s,
    partials, tol, maxit);
  if(cudaPeekAtLastError() != cudaSuccess) return BBB_ERR_CUDA;
  int cur = 0, batch = 1, total = 0;
  for(;;) {
    for(int q = 0; q < batch; q++) {
      k_bicgA<double, V><<<grd, blk, 0, st>>>(B, O, mask, sv, tv, pp[cur],
        vv[cur], rh, r, pp[cur ^ 1], vv[cur ^ 1], x, s, partials);
      k_bicgB<double, V><<<grd, blk, 0, st>>>(B, O, mask, r, vv[cur ^ 1], rh,
        sv, tv, s, partials);
      cur ^= 1;
    }
    total += batch;
    if(cudaMemcpyAsync(h, s, sizeof(bbb_kry), cudaMemcpyDeviceToHost, st)
      != cudaSuccess) return BBB_ERR_CUDA;
    if(cudaStreamSynchronize(st) != cudaSuccess) return BBB_ERR_CUDA;
    if(h->done || total > maxit + 4) break;
    if(batch < 16) batch *= 2;
  }
  return BBB_OK;
}

extern "C" int bbb_PP_bicgstab_static(int nx, int ny, int nz, double dx,
  double dy, double dz, int perx, int pery, int perz, const double *u_star_d,
  const double *v_star_d, const double *w_star_d, const int *phase_d,
  const int *flag_u_d, const int *flag_v_d, const int *flag_w_d,
  double rho_f_, double dt_, double tol, int maxit, double *phi_d,
  int *iters, double *resid, void *stream)
{
  if(nx < 1 || ny < 1 || nz < 1) return BBB_ERR_CONFIG;
  long long n = (long long)nx * ny * nz;
  if(n > BBB_STATIC_MAX_CELLS) return BBB_ERR_TOO_LARGE;
  int dev = 0;
  if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return BBB_ERR_CUDA;
  unsigned char *base;
  {
    std::lock_guard<std::mutex> hold(g_static_lock);
    if(!g_static_addr[dev]) {
      unsigned char *p = NULL;
      if(cudaGetSymbolAddress((void **)&p, g_static_scratch) != cudaSuccess || !p)
        return BBB_ERR_CUDA;
      g_static_addr[dev] = p;
    }
    base = g_static_addr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  /* carve the scratch */
  long long off = 0;
#define CARVE(T, ptr, bytes) do { ptr = (T *)(base + off); \
  off += 256LL * (((long long)(bytes) + 255LL) / 256LL); } while(0)
  bbb_kry *s; double *partials; uint8_t *mask;
  double *b, *x, *r, *rh, *pp[2], *vv[2], *sv, *tv;
  CARVE(bbb_kry, s, 256);
  CARVE(double, partials, BBB_STATIC_PARTIALS * 8LL);
  CARVE(uint8_t, mask, BBB_STATIC_MAX_CELLS);
  size_t vb = (size_t)BBB_STATIC_MAX_CELLS * 8;
  CARVE(double, b, vb); CARVE(double, x, vb); CARVE(double, r, vb);
  CARVE(double, rh, vb); CARVE(double, pp[0], vb); CARVE(double, pp[1], vb);
  CARVE(double, vv[0], vb); CARVE(double, vv[1], vb); CARVE(double, sv, vb);
  CARVE(double, tv, vb);
#undef CARVE
  /* geometry of the reference's ghosted layouts */
  bbb_geom G;
  memset(&G, 0, sizeof(G));
  G.nx = nx; G.ny = ny; G.nz = nz;
  G.cc_s1 = nx + 2; G.cc_s2 = (nx + 2) * (ny + 2);
  G.fx_s1 = nx + 3; G.fx_s2 = (nx + 3) * (ny + 2);
  G.fy_s1 = nx + 2; G.fy_s2 = (nx + 2) * (ny + 3);
  G.fz_s1 = nx + 2; G.fz_s2 = (nx + 2) * (ny + 2);
  G.dx = dx; G.dy = dy; G.dz = dz;
  int V = pick_vec(nx, sizeof(double));
  int per_sm = V == 2 ? bicg_per_sm<double, 2>() : bicg_per_sm<double, 1>();
  boxc B = make_box(nx, ny, nz, perx, pery, perz, 0, 0, 0, V, per_sm);
  dim3 grd = box_grid(B);
  if((long long)grd.x * grd.y * grd.z * 5 > BBB_STATIC_PARTIALS) return BBB_ERR_TOO_LARGE;
  opc O;
  O.wx = 1. / (dx * dx); O.wy = 1. / (dy * dy); O.wz = 1. / (dz * dz);
  O.helm = 0;
  /* the reduction ticket and the scalars start from zero on every call */
  if(cudaMemsetAsync(s, 0, sizeof(bbb_kry), st) != cudaSuccess) return BBB_ERR_CUDA;
  k_mask_p<<<NPW, 256, 0, st>>>(flag_u_d, flag_v_d, flag_w_d, phase_d, G, mask);
  k_pp_rhs<<<NPW, 256, 0, st>>>(u_star_d, v_star_d, w_star_d, phi_d, phase_d,
    G, rho_f_ / dt_, b, x, s, partials);
  bbb_kry h;
  int rc = V == 2
    ? static_iterations<2>(B, O, mask, b, x, r, rh, pp, vv, sv, tv, s,
        partials, tol, maxit, st, &h)
    : static_iterations<1>(B, O, mask, b, x, r, rh, pp, vv, sv, tv, s,
        partials, tol, maxit, st, &h);
  if(rc != BBB_OK) return rc;
  k_pp_writeback<<<NPW, 256, 0, st>>>(x, phi_d, G, s);
  if(cudaMemcpyAsync(&h, s, sizeof(bbb_kry), cudaMemcpyDeviceToHost, st)
    != cudaSuccess) return BBB_ERR_CUDA;
  if(cudaStreamSynchronize(st) != cudaSuccess) return BBB_ERR_CUDA;
  if(iters) *iters = h.iter;
  if(resid) *resid = h.bnorm > 0 ? h.rnorm / h.bnorm : h.rnorm;
  if(h.status == BBB_ERR_NONFINITE) return BBB_ERR_NONFINITE;
  return h.converged ? BBB_OK : BBB_ERR_NOT_CONVERGED;
}
