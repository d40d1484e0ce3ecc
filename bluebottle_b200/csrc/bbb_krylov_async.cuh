/* bbb_krylov_async.cuh -- the two BiCGSTAB passes, the FP64 outer residual
 * of the defect correction and the Helmholtz CG stencil pass with their
 * inputs staged by the tensor memory accelerator (included by
 * bbb_krylov.cu, which defines boxc, opc, optab, op_apply, mapx/y/z, lin
 * and the reductions).
 *
 * Same arithmetic as k_bicgA / k_bicgB / k_outer_resid / k_cg1, for rows
 * of a multiple of 128 cells, with one difference in where a value lives:
 * pass B does not store s = r - alpha v; pass A forms it again from the r
 * and v it reads anyway (the same FP32 or FP64 expression, so the same
 * bits), which takes one vector write out of every iteration.  Pass A
 * reads r and writes the new r, so r alternates between two buffers (the
 * second is the one s would have used).  A block owns a tile of 128 cells
 * x TH rows (TH = 8 or 16, per pass and precision) and marches along z.
 * For every plane it needs, one thread issues a handful of 3-D tensor
 * copies -- per input array one box of TH + 2 rows x (128 + two 16-byte
 * x-halo chunks), the mask likewise, the block's own TH rows of the arrays
 * only it reads -- into a shared-memory stage whose mbarrier completes when
 * all bytes have landed.
 * NS stages rotate, so the next plane is in flight while the block
 * computes this one (two stages measured faster than three, four or five
 * on 256x256x512: pass A 2%, pass B 5%, the FP64 pass B 7%); the warps
 * synchronise only through the stages' barriers and release counts, never
 * block-wide inside a run of planes.
 *
 * Every warp owns R adjacent tile rows (R = 1 or 2) and computes the
 * Jacobi-scaled stencil input q for its rows and for the rows just south
 * and north of them straight from the stage (no shared ring, so the stages
 * of two blocks fit per SM); the rows' x-halo q come from the stage's halo
 * chunks.  A plane's stencil
 * sum is formed up to its top term as soon as its stage is read, so its
 * south / north q die at once; the plane's q, that partial sum and its
 * epilogue inputs stay in registers until the plane above completes it.
 *
 * Wrap-around neighbours that a tiled box cannot express land in slots of
 * their own, never under a box (two asynchronous writes to one byte would
 * race): the rows y = -1 and y = ny (the box's wS / wN rows) as plain bulk
 * copies of the tile's 128 cells, and the x-halo chunks at x = -1 and
 * x = nx (holding cells wW / wE) as 16-byte-wide boxes of the tile's TH
 * rows.  The tiled boxes' out-of-range parts are zero-filled and never read.
 *
 * Waits on the stage barriers are bounded; a wait that runs out marks the
 * solve failed (status BBB_ERR_CUDA through the scalars) and the kernel
 * carries on without reading past its buffers. */
#ifndef BBB_KRYLOV_ASYNC_CUH
#define BBB_KRYLOV_ASYNC_CUH

#include <cuda.h>

#define AS_W 128
#define AS_THREADS 256
/* pipeline stages and resident blocks per SM of each pass (F: FP32, D:
 * FP64; 0 pass A, 1 pass B, 2 the FP64 outer residual, 3 the Helmholtz
 * CG stencil pass); build-time switches for measurement */
#ifndef BBB_AS_NS_F0
#define BBB_AS_NS_F0 2
#endif
#ifndef BBB_AS_NS_F1
#define BBB_AS_NS_F1 2
#endif
#ifndef BBB_AS_NS_D0
#define BBB_AS_NS_D0 2
#endif
#ifndef BBB_AS_NS_D1
#define BBB_AS_NS_D1 2
#endif
#ifndef BBB_AS_NS_D2
#define BBB_AS_NS_D2 2
#endif
#ifndef BBB_AS_NS_F3
#define BBB_AS_NS_F3 2
#endif
#ifndef BBB_AS_NS_D3
#define BBB_AS_NS_D3 2
#endif
#ifndef BBB_AS_MINB_F3
#define BBB_AS_MINB_F3 2
#endif
#ifndef BBB_AS_MINB_D3
#define BBB_AS_MINB_D3 3
#endif
#ifndef BBB_AS_MINB_F0
#define BBB_AS_MINB_F0 2
#endif
#ifndef BBB_AS_MINB_F1
#define BBB_AS_MINB_F1 2
#endif
#ifndef BBB_AS_MINB_D0
#define BBB_AS_MINB_D0 1
#endif
#ifndef BBB_AS_MINB_D1
#define BBB_AS_MINB_D1 2
#endif
#ifndef BBB_AS_MINB_D2
#define BBB_AS_MINB_D2 3
#endif
/* rows per warp (R) and tile height (TH, a multiple of R: the block has
 * TH / R warps) of pass B, the CG stencil pass and the outer residual;
 * pass A keeps one row per warp and 8-row tiles.  FP32 pass B and CG run
 * two rows per warp in 16-row tiles (128 registers, 2 blocks per SM): on
 * 256x256x512 pass B 0.178 -> 0.150 ms, CG 0.149 -> 0.146 ms against one
 * row per warp in 8-row tiles (80 registers, 3 blocks per SM).  FP64 pass
 * B, CG and the outer residual run two rows per warp in 8-row tiles (4
 * warps; 248 / 168 / 168 registers, 2 / 3 / 3 blocks per SM): pass B
 * 0.297 -> 0.284 ms, CG 0.250 -> 0.234 ms, outer residual 0.182 -> 0.167
 * ms against one row per warp with 8 warps */
#ifndef BBB_AS_R_F1
#define BBB_AS_R_F1 2
#endif
#ifndef BBB_AS_TH_F1
#define BBB_AS_TH_F1 16
#endif
#ifndef BBB_AS_R_D1
#define BBB_AS_R_D1 2
#endif
#ifndef BBB_AS_TH_D1
#define BBB_AS_TH_D1 8
#endif
#ifndef BBB_AS_R_F3
#define BBB_AS_R_F3 2
#endif
#ifndef BBB_AS_TH_F3
#define BBB_AS_TH_F3 16
#endif
#ifndef BBB_AS_R_D2
#define BBB_AS_R_D2 2
#endif
#ifndef BBB_AS_TH_D2
#define BBB_AS_TH_D2 8
#endif
#ifndef BBB_AS_R_D3
#define BBB_AS_R_D3 2
#endif
#ifndef BBB_AS_TH_D3
#define BBB_AS_TH_D3 8
#endif

__host__ __device__ constexpr int as_rup(int v, int a) { return (v + a - 1) / a * a; }

/* Stage layout in bytes (T the element type, CH = 16 / sizeof(T), TH the
 * tile height in rows):
 *   per halo array (pass A: r, t, p, v; pass B: r, v; outer residual: x;
 *   CG: r, p) a region of
 *     TH + 2 box rows of [CH | 128 | CH] cells (tile rows j0-1 .. j0+TH),
 *     2 extra rows of 128 cells (y = -1, y = ny);
 *   mask: TH + 2 rows of [16 | 128 | 16] bytes, 2 extra rows of 128;
 *   own arrays (pass A: x, rh; pass B: rh; outer residual: b; CG: none):
 *   TH rows of 128 cells;
 *   x-wrap chunks: per halo array and the mask [2 sides][TH rows][16 B].
 * Regions start on 128-byte boundaries (tensor-copy destinations). */
template <typename T, int PASS>
struct as_layout {
  static constexpr int ESZ = (int)sizeof(T);
  static constexpr int CH = 16 / ESZ;
  static constexpr int NA = PASS == 0 ? 4 : (PASS == 1 || PASS == 3 ? 2 : 1);
  static constexpr int NO = PASS == 0 ? 2 : (PASS == 3 ? 0 : 1);
  /* rows per warp, tile rows, warps and threads per block */
  static constexpr int R = ESZ == 4
    ? (PASS == 1 ? BBB_AS_R_F1 : (PASS == 3 ? BBB_AS_R_F3 : 1))
    : (PASS == 1 ? BBB_AS_R_D1 : (PASS == 3 ? BBB_AS_R_D3
       : (PASS == 2 ? BBB_AS_R_D2 : 1)));
  static constexpr int TH = ESZ == 4
    ? (PASS == 1 ? BBB_AS_TH_F1 : (PASS == 3 ? BBB_AS_TH_F3 : 8))
    : (PASS == 1 ? BBB_AS_TH_D1 : (PASS == 3 ? BBB_AS_TH_D3
       : (PASS == 2 ? BBB_AS_TH_D2 : 8)));
  static constexpr int WARPS = TH / R;
  static constexpr int THREADS = 32 * WARPS;
  static_assert(TH % R == 0 && WARPS >= 1 && WARPS <= 32 && TH + 2 <= 256,
                "tile height: a multiple of the rows per warp, 1..32 warps");
  static constexpr int BOXW = AS_W + 2 * CH;        /* halo-array box  */
  static constexpr int BOXH = TH + 2;
  static constexpr int MBOXW = AS_W + 32;            /* mask box        */
  static constexpr int ROWP = BOXW * ESZ;
  static constexpr int OWNB = AS_W * ESZ;
  static constexpr int EXT_OFF = BOXH * ROWP;
  static constexpr int AREG = as_rup(EXT_OFF + 2 * OWNB, 128);
  static constexpr int MROWP = MBOXW;
  static constexpr int MEXT_OFF = BOXH * MROWP;
  static constexpr int MREG = as_rup(MEXT_OFF + 2 * 128, 128);
  static constexpr int MASK_OFF = NA * AREG;
  static constexpr int OWN_OFF = MASK_OFF + MREG;
  static constexpr int XW_OFF = OWN_OFF + NO * TH * OWNB;
  /* x-wrap chunks of one array: 2 sides x TH rows x 16 bytes */
  static constexpr int XWA = 2 * TH * 16;
  static constexpr int STAGE = as_rup(XW_OFF + (NA + 1) * XWA, 128);
  /* stages in the ring */
  static constexpr int NS = ESZ == 4
    ? (PASS == 0 ? BBB_AS_NS_F0 : (PASS == 3 ? BBB_AS_NS_F3 : BBB_AS_NS_F1))
    : (PASS == 0 ? BBB_AS_NS_D0 : (PASS == 1 ? BBB_AS_NS_D1
       : (PASS == 3 ? BBB_AS_NS_D3 : BBB_AS_NS_D2)));
  static constexpr int TAB_OFF = NS * STAGE;
  static constexpr int BAR_OFF = TAB_OFF + 2 * 128 * ESZ;
  static constexpr int CNT_OFF = BAR_OFF + NS * 8;      /* release counts */
  static constexpr int SH_OFF = as_rup(CNT_OFF + NS * 4, 16);
  /* + 128: the dynamic window is aligned up to 128 bytes at run time */
  static constexpr int SMEM = SH_OFF + 32 * 5 * 8 + 128;
  /* resident blocks per SM the register budget targets */
  static constexpr int MINB = ESZ == 4
    ? (PASS == 0 ? BBB_AS_MINB_F0 : (PASS == 3 ? BBB_AS_MINB_F3 : BBB_AS_MINB_F1))
    : (PASS == 0 ? BBB_AS_MINB_D0 : (PASS == 1 ? BBB_AS_MINB_D1
       : (PASS == 3 ? BBB_AS_MINB_D3 : BBB_AS_MINB_D2)));
  /* plane-aligned group runs (retile): off -- grouping neighbouring tiles
   * gets the same L2 reuse without idle slots */
  static constexpr bool ALIGN = false;
  /* bytes a stage receives: the boxes always, the wrap slots at edges */
  static constexpr int TX_BASE = NA * BOXH * ROWP + BOXH * MROWP + NO * TH * OWNB;
  static constexpr int TX_XSIDE = (NA + 1) * TH * 16;
  static constexpr int TX_YSIDE = NA * OWNB + 128;
};

/* the tensor maps of one pass, passed by value as a grid constant */
struct as_maps {
  CUtensorMap h[4];     /* halo arrays, box {128 + 2 CH, TH + 2, 1}    */
  CUtensorMap hx[4];    /* halo arrays, box {CH, TH, 1}                */
  CUtensorMap m, mx;    /* mask, boxes {160, TH + 2, 1} and {16, TH, 1} */
  CUtensorMap o[2];     /* own arrays, box {128, TH, 1}                */
};

/* the global arrays of one pass */
template <typename T>
struct as_args {
  const uint8_t *mask;
  const T *h[4];          /* halo arrays                                 */
  T *w0, *w1, *w2;        /* pass A: r_new, p_new, v_new; pass B: -, t;
                             CG: p_new, y = A p_new                     */
  T *x;                   /* pass A: x, updated in place                 */
  bbb_kry *s;
  double *partials;
  /* outer residual (pass 2): r = b - A x rounded to FP32, and the inner
   * solve's scalars it sets up */
  float *rf;
  bbb_kry *si;
  double itol;
  int imaxit, project;
  long long n;
};

__device__ __forceinline__ uint32_t as_saddr(const void *p)
{ return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void as_bar_init(uint32_t bar)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar) : "memory");
}

__device__ __forceinline__ void as_expect(uint32_t bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(bar), "r"(bytes) : "memory");
}

/* contiguous bulk copy global -> shared (16-byte aligned, 16-byte multiple) */
__device__ __forceinline__ void as_copy(uint32_t dst, const void *src,
  uint32_t bytes, uint32_t bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
               " [%0], [%1], %2, [%3];"
               :: "r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}

/* 3-D tiled tensor copy of the box at (x, y, z); x * element size is a
 * multiple of 16 bytes at every call site */
__device__ __forceinline__ void as_box(uint32_t dst, const CUtensorMap *map,
  int x, int y, int z, uint32_t bar)
{
  asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile"
               ".mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
               :: "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y),
                  "r"(z), "r"(bar) : "memory");
}

/* bounded wait for the phase of parity `par`; false when the limit ran
 * out.  Each try may suspend the thread for up to 20 us until the phase
 * completes, so waiting warps do not spin on the issue slots; the bound is
 * 2^16 tries.  (try_wait with the hardware's default time limit measured
 * the same on 256x256x512, polling test_wait 2-5% slower.) */
__device__ __forceinline__ bool as_wait(uint32_t bar, uint32_t par)
{
  for(int it = 0; it < (1 << 16); it++) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(ok) : "r"(bar), "r"(par), "r"(20000) : "memory");
    if(ok) return true;
  }
  return false;
}

/* one warp's release of a stage: acquire-release add on the stage's count
 * (orders the warp's reads of the stage before the refill its last
 * releaser issues); returns the count before the add */
__device__ __forceinline__ uint32_t as_release(uint32_t cnt)
{
  uint32_t old;
  asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], 1;"
               : "=r"(old) : "r"(cnt) : "memory");
  return old;
}

/* where a tile touches the box's faces */
struct as_edges {
  int xl, xr, ys, yn;     /* i0 == 0, i0 + 128 == nx, j0 == 0, j0 + TH >= ny */
};

template <int TH>
__device__ __forceinline__ as_edges as_tile_edges(const boxc &B, int i0, int j0)
{
  as_edges e;
  e.xl = i0 == 0;
  e.xr = i0 + AS_W == B.nx;
  e.ys = j0 == 0;
  e.yn = j0 + TH >= B.ny;
  return e;
}

/* Issue the copies of plane gk of tile (i0, j0) into the stage at shared
 * address st (one thread; it arms the barrier with the byte count first). */
template <typename T, int PASS>
__device__ __forceinline__ void as_issue(const boxc &B, const as_args<T> &A,
  const as_maps &M, uint32_t st, uint32_t bar, int i0, int j0, int gk,
  const as_edges &E)
{
  typedef as_layout<T, PASS> L;
  uint32_t tx = L::TX_BASE + (uint32_t)(E.xl + E.xr) * L::TX_XSIDE
    + (uint32_t)(E.ys + E.yn) * L::TX_YSIDE;
  as_expect(bar, tx);
#pragma unroll
  for(int a = 0; a < L::NA; a++)
    as_box(st + a * L::AREG, &M.h[a], i0 - (L::BOXW - AS_W) / 2,
      j0 - (L::BOXH - L::TH) / 2, gk, bar);
  as_box(st + L::MASK_OFF, &M.m, i0 - (L::MBOXW - AS_W) / 2, j0 - (L::BOXH - L::TH) / 2,
    gk, bar);
#pragma unroll
  for(int b = 0; b < L::NO; b++)
    as_box(st + L::OWN_OFF + b * L::TH * L::OWNB, &M.o[b], i0, j0, gk, bar);
  for(int side = 0; side < 2; side++) {
    if(side == 0 ? !E.xl : !E.xr) continue;
    int g = side == 0 ? B.wW : B.wE;
    uint32_t d = st + L::XW_OFF + side * L::TH * 16;
#pragma unroll
    for(int a = 0; a < L::NA; a++)
      as_box(d + a * L::XWA, &M.hx[a], g / L::CH * L::CH, j0, gk, bar);
    as_box(d + L::NA * L::XWA, &M.mx, g / 16 * 16, j0, gk, bar);
  }
  for(int side = 0; side < 2; side++) {
    if(side == 0 ? !E.ys : !E.yn) continue;
    long long c = lin(B, i0, side == 0 ? B.wS : B.wN, gk);
#pragma unroll
    for(int a = 0; a < L::NA; a++)
      as_copy(st + a * L::AREG + L::EXT_OFF + side * L::OWNB, A.h[a] + c,
        L::OWNB, bar);
    as_copy(st + L::MASK_OFF + L::MEXT_OFF + side * 128, A.mask + c, 128, bar);
  }
}

template <typename T>
__device__ __forceinline__ void as_ld4(const uint8_t *p, T (&o)[4])
{
  if constexpr(sizeof(T) == 4) {
    float4 v = *reinterpret_cast<const float4 *>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  } else {
    double2 a = reinterpret_cast<const double2 *>(p)[0];
    double2 b = reinterpret_cast<const double2 *>(p)[1];
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
  }
}

template <typename T>
__device__ __forceinline__ void as_st4(T *p, const T (&v)[4])
{
  if constexpr(sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
  }
}

/* r += sum of a[v] * b[v] over 4 cells: exact FP64 products (FP32
 * operands widen exactly) summed one by one, the order of the register
 * kernels.  (Fusing the 4 FP32 products in FP32 first saves a few
 * instructions but cost the FP32 inner solves 3% more iterations.) */
template <typename T>
__device__ __forceinline__ void as_dot4(double &r, const T (&a)[4], const T (&b)[4])
{
#pragma unroll
  for(int v = 0; v < 4; v++) r += (double)a[v] * (double)b[v];
}

template <typename T>
__device__ __forceinline__ void as_sum4(double &r, const T (&a)[4])
{
#pragma unroll
  for(int v = 0; v < 4; v++) r += (double)a[v];
}

/* (A q) at one cell, as op_apply (same terms in the same order), with the
 * face terms of clear mask bits skipped rather than multiplied by zero --
 * the same value for finite q; w* already carry the operator's sign.  Split
 * in two so a plane's sum is formed while its own neighbour rows are at
 * hand: as_apply_lo sums the terms B, S, W, C, E, N; as_apply_hi adds T
 * once the plane above is staged, then applies the inside-particle rule. */
template <typename T>
__device__ __forceinline__ T as_apply_lo(unsigned m, T d, T wx, T wy, T qB,
  T qS, T qW, T qC, T qE, T qN, T wz)
{
  T acc = (T)0.;
  if(m & BBB_MB) acc += wz * qB;
  if(m & BBB_MS) acc += wy * qS;
  if(m & BBB_MW) acc += wx * qW;
  acc += d * qC;
  if(m & BBB_ME) acc += wx * qE;
  if(m & BBB_MN) acc += wy * qN;
  return acc;
}

template <typename T>
__device__ __forceinline__ T as_apply_hi(unsigned m, T wz, T acc, T qC, T qT)
{
  if(m & BBB_MT) acc += wz * qT;
  return (m & BBB_MID) ? qC : acc;
}

/* pass scalars, read once per kernel */
struct as_scal {
  double alpha, omega, beta, bo;
  int first;
};

/* The Helmholtz CG direction at 4 cells (pass 3): p = M r + beta p_old
 * (r array 0, p_old array 1 at h + stride), or p_old itself in the first
 * iteration, where the set-up left p = M r -- the expression of prod_c1 */
template <typename T>
__device__ __forceinline__ void as_cg_q4(const uint8_t *h, int stride,
  unsigned mw, const T *dinv, const as_scal &S, T (&q)[4])
{
  as_ld4<T>(h + stride, q);
  if(!S.first) {
    T rr[4];
    const T be = (T)S.beta;
    as_ld4<T>(h, rr);
#pragma unroll
    for(int a = 0; a < 4; a++) q[a] = (T)1. * (dinv[mbyte(mw, a)] * rr[a]) + be * q[a];
  }
}

/* q at 4 consecutive cells of a staged row: h the first cell of array 0
 * (array a at h + a * AREG), mw the 4 mask bytes */
template <typename T, int PASS>
__device__ __forceinline__ void as_q4(const uint8_t *h, unsigned mw,
  const T *dinv, const as_scal &S, T (&q)[4])
{
  typedef as_layout<T, PASS> L;
  if constexpr(PASS == 0) {
    T ss[4];
    as_ld4<T>(h, ss);
    if(S.first) {
#pragma unroll
      for(int a = 0; a < 4; a++) q[a] = dinv[mbyte(mw, a)] * ss[a];
    } else {
      T tt[4], pp[4], vv[4];
      T al = (T)S.alpha, om = (T)S.omega, be = (T)S.beta, bo = (T)S.bo;
      as_ld4<T>(h + 1 * L::AREG, tt);
      as_ld4<T>(h + 2 * L::AREG, pp);
      as_ld4<T>(h + 3 * L::AREG, vv);
#pragma unroll
      for(int a = 0; a < 4; a++) {
        ss[a] = ss[a] - al * vv[a];        /* s = r - alpha v, as pass B */
        T rr = ss[a] - om * tt[a];
        T pn = rr + be * pp[a] + bo * vv[a];
        q[a] = dinv[mbyte(mw, a)] * pn;
      }
    }
  } else if constexpr(PASS == 1) {
    T rr[4], vv[4];
    T al = (T)S.alpha;
    as_ld4<T>(h, rr);
    as_ld4<T>(h + 1 * L::AREG, vv);
#pragma unroll
    for(int a = 0; a < 4; a++) q[a] = dinv[mbyte(mw, a)] * (rr[a] - al * vv[a]);
  } else if constexpr(PASS == 3) {
    as_cg_q4<T>(h, L::AREG, mw, dinv, S, q);
  } else {
    as_ld4<T>(h, q);                   /* outer residual: q = x */
    (void)mw; (void)dinv; (void)S;
  }
}

/* The block's own 4 cells of a staged row: q, and the pass's pointwise
 * work -- stores at global index gc, sums into red.  o is the cells' first
 * own-array entry (pass A: x at o, rh at o + TH rows; pass B: rh at o);
 * raw0 / raw1 carry what the epilogue needs (pass A: rh; pass B: s, rh). */
template <typename T, int PASS>
__device__ __forceinline__ void as_own4(const uint8_t *h, unsigned mw,
  const uint8_t *o, const T *dinv, const as_scal &S, long long gc,
  const as_args<T> &A, T (&q)[4], T (&raw0)[4], T (&raw1)[4], double (&red)[5])
{
  typedef as_layout<T, PASS> L;
  if constexpr(PASS == 0) {
    T ss[4], rr[4], pn[4];
    as_ld4<T>(h, ss);
    if(S.first) {
#pragma unroll
      for(int a = 0; a < 4; a++) { rr[a] = ss[a]; pn[a] = rr[a]; }
    } else {
      T tt[4], pp[4], vv[4], xx[4];
      T al = (T)S.alpha, om = (T)S.omega, be = (T)S.beta, bo = (T)S.bo;
      as_ld4<T>(h + 1 * L::AREG, tt);
      as_ld4<T>(h + 2 * L::AREG, pp);
      as_ld4<T>(h + 3 * L::AREG, vv);
      as_ld4<T>(o, xx);
#pragma unroll
      for(int a = 0; a < 4; a++) {
        ss[a] = ss[a] - al * vv[a];        /* s = r - alpha v, as pass B */
        rr[a] = ss[a] - om * tt[a];
        pn[a] = rr[a] + be * pp[a] + bo * vv[a];
        T di = dinv[mbyte(mw, a)];
        xx[a] = xx[a] + al * (di * pp[a]) + om * (di * ss[a]);
      }
      as_sum4<T>(red[3], xx);
      as_st4<T>(A.x + gc, xx);
    }
#pragma unroll
    for(int a = 0; a < 4; a++) q[a] = dinv[mbyte(mw, a)] * pn[a];
    as_ld4<T>(o + L::TH * L::OWNB, raw0);
    as_dot4<T>(red[1], rr, rr);
    as_dot4<T>(red[2], raw0, rr);
    as_st4<T>(A.w0 + gc, rr);
    as_st4<T>(A.w1 + gc, pn);
  } else if constexpr(PASS == 1) {
    T rr[4], vv[4];
    T al = (T)S.alpha;
    as_ld4<T>(h, rr);
    as_ld4<T>(h + 1 * L::AREG, vv);
#pragma unroll
    for(int a = 0; a < 4; a++) {
      raw0[a] = rr[a] - al * vv[a];
      q[a] = dinv[mbyte(mw, a)] * raw0[a];
    }
    as_ld4<T>(o, raw1);
    as_dot4<T>(red[2], raw0, raw0);
  } else if constexpr(PASS == 3) {
    /* Helmholtz CG: the new direction p is stored (w0) and kept for the
     * epilogue's (p, A p) */
    as_cg_q4<T>(h, L::AREG, mw, dinv, S, q);
#pragma unroll
    for(int a = 0; a < 4; a++) raw0[a] = q[a];
    as_st4<T>(A.w0 + gc, q);
    (void)o; (void)raw1; (void)red;
  } else {
    /* outer residual: q = x (sum x over the owned cells), raw0 = b */
    as_ld4<T>(h, q);
    as_sum4<T>(red[1], q);
    as_ld4<T>(o, raw0);
    (void)mw; (void)dinv; (void)S; (void)gc; (void)A; (void)raw1;
  }
}

/* q at one x-halo cell: h its array-0 entry, arrays `stride` bytes apart,
 * m its mask byte */
template <typename T, int PASS>
__device__ __forceinline__ T as_q1(const uint8_t *h, int stride, unsigned m,
  const T *dinv, const as_scal &S)
{
  if constexpr(PASS == 0) {
    T ss = *reinterpret_cast<const T *>(h);
    T pn;
    if(S.first) pn = ss;
    else {
      T tt = *reinterpret_cast<const T *>(h + 1 * stride);
      T pp = *reinterpret_cast<const T *>(h + 2 * stride);
      T vv = *reinterpret_cast<const T *>(h + 3 * stride);
      ss = ss - (T)S.alpha * vv;            /* s = r - alpha v, as pass B */
      T rr = ss - (T)S.omega * tt;
      pn = rr + (T)S.beta * pp + (T)S.bo * vv;
    }
    return dinv[m] * pn;
  } else if constexpr(PASS == 1) {
    T rr = *reinterpret_cast<const T *>(h);
    T vv = *reinterpret_cast<const T *>(h + stride);
    return dinv[m] * (rr - (T)S.alpha * vv);
  } else if constexpr(PASS == 3) {
    T pp = *reinterpret_cast<const T *>(h + stride);
    if(S.first) return pp;
    T rr = *reinterpret_cast<const T *>(h);
    return (T)1. * (dinv[m] * rr) + (T)S.beta * pp;
  } else {
    (void)stride; (void)m; (void)dinv; (void)S;
    return *reinterpret_cast<const T *>(h);
  }
}

/* One staged pass (PASS 0: BiCGSTAB pass A, 1: pass B, 2: the FP64 outer
 * residual of the defect correction, 3: the Helmholtz CG stencil pass) over
 * this block's units, TH / R warps, warp w owning the R adjacent tile rows
 * R w .. R w + R - 1, lane l cells 4l..4l+3 of each.
 * Per plane: wait for the stage; each warp forms q of its rows (with the
 * pointwise work where the plane is the block's), of the rows just south
 * and north of them and of their x-halo cells; releases the stage (the
 * last warp to release it refills it with the plane NS ahead); then the
 * stencil of this plane up to its top term and the epilogue of the plane
 * below, from registers.  With R > 1 a warp's own rows are each other's
 * south / north neighbours, so q is formed R + 2 times per R rows instead
 * of 3 times per row. */
template <typename T, int PASS>
__global__ void __launch_bounds__(as_layout<T, PASS>::THREADS, as_layout<T, PASS>::MINB)
k_bicg_async(boxc B, opc O, as_args<T> A, const __grid_constant__ as_maps M)
{
  typedef as_layout<T, PASS> L;
  constexpr int R = L::R, NW = L::WARPS;
  bbb_kry *s = A.s;
  if(((volatile bbb_kry *)s)->done) return;
  extern __shared__ __align__(128) uint8_t as_dyn[];
  /* aligned by an offset into the shared array (not by pointer masking),
   * so every access below stays a shared-space access */
  uint8_t *sm = as_dyn + ((128u - (as_saddr(as_dyn) & 127u)) & 127u);
  optab<T> &tab = *reinterpret_cast<optab<T> *>(sm + L::TAB_OFF);
  uint64_t *bars = reinterpret_cast<uint64_t *>(sm + L::BAR_OFF);
  double *sh = reinterpret_cast<double *>(sm + L::SH_OFF);
  const uint32_t sbase = as_saddr(sm);
  const int tid = threadIdx.x, tx = tid & 31, w = tid >> 5;
  uint32_t *rel = reinterpret_cast<uint32_t *>(sm + L::CNT_OFF);
  if(tid == 0) {
    for(int b = 0; b < L::NS; b++) { as_bar_init(as_saddr(&bars[b])); rel[b] = 0u; }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  optab_fill<T>(tab, O);                  /* ends with a barrier */
  as_scal S;
  S.alpha = s->alpha; S.omega = s->omega; S.beta = s->beta;
  S.bo = -S.beta * S.omega; S.first = s->first;
  const T sg = O.helm ? (T)-1. : (T)1.;
  const T wx = (T)O.wx * sg, wy = (T)O.wy * sg, wz = (T)O.wz * sg;
  double red[5] = {0., 0., 0., 0., 0.};
  int bad = 0;
  long long nload = 0;
  /* this block's group, its tile inside the group, the group's units */
  const int G = B.gx * B.gy;
  const long long grp = blockIdx.x / G;
  const int mem = (int)(blockIdx.x % G);
  long long u0 = grp * B.q + (grp < B.r ? grp : B.r);
  const long long u1 = u0 + B.q + (grp < B.r ? 1 : 0);
  const int gtx = B.tiles_x / B.gx;     /* groups along x */
  const int col = tx * 4;
  while(u0 < u1) {
    const long long gt = u0 / B.nz;
    const int k0 = (int)(u0 - gt * B.nz);
    const long long left_ = u1 - u0;
    const int k1 = left_ < (long long)(B.nz - k0) ? k0 + (int)left_ : B.nz;
    const int ti = (int)(gt % gtx) * B.gx + mem % B.gx;
    const int tj = (int)(gt / gtx) * B.gy + mem / B.gx;
    const int i0 = ti * AS_W, j0 = tj * L::TH;
    /* the warp's first row, its rows inside the box (<= 0: none) and the
     * box row of its first row */
    const int jw = j0 + R * w;
    const int nv = B.ny - jw < R ? B.ny - jw : R;
    const int rb = R * w + 1;
    const as_edges E = as_tile_edges<L::TH>(B, i0, j0);
    const int cnt = k1 - k0 + 2;
    const long long L0 = nload;
    if(tid == 0)
      for(int a = 0; a < L::NS && a < cnt; a++) {
        int b = (int)((L0 + a) % L::NS);
        as_issue<T, PASS>(B, A, M, sbase + b * L::STAGE, as_saddr(&bars[b]), i0, j0,
          mapz(B, k0 - 1 + a), E);
      }
    /* this warp's offsets inside a stage: its first own row (box row rb;
     * row r at + r ROWP), the row south of its first row (box row rb - 1
     * or the wrap row at the face), the row north of its last row inside
     * the box (box row rb + R or the wrap row), the x-halo cell of its
     * first row (lane 0 west, lane 31 east; row r at + r hx_rs) */
    const int h_own = rb * L::ROWP + (L::CH + col) * L::ESZ;
    const int m_own = L::MASK_OFF + rb * L::MROWP + 16 + col;
    const int h_s = jw == 0 ? L::EXT_OFF + col * L::ESZ
                            : (rb - 1) * L::ROWP + (L::CH + col) * L::ESZ;
    const int m_s = jw == 0 ? L::MASK_OFF + L::MEXT_OFF + col
                            : L::MASK_OFF + (rb - 1) * L::MROWP + 16 + col;
    const bool nwrap = jw + nv == B.ny;
    const int h_n = nwrap ? L::EXT_OFF + L::OWNB + col * L::ESZ
                          : (rb + R) * L::ROWP + (L::CH + col) * L::ESZ;
    const int m_n = nwrap ? L::MASK_OFF + L::MEXT_OFF + 128 + col
                          : L::MASK_OFF + (rb + R) * L::MROWP + 16 + col;
    int h_x, m_x, x_stride, hx_rs, mx_rs;
    if(tx == 0) {
      if(E.xl) {
        h_x = L::XW_OFF + (R * w) * 16 + (B.wW % L::CH) * L::ESZ;
        m_x = L::XW_OFF + L::NA * L::XWA + (R * w) * 16 + B.wW % 16;
        x_stride = L::XWA; hx_rs = 16; mx_rs = 16;
      } else {
        h_x = rb * L::ROWP + (L::CH - 1) * L::ESZ;
        m_x = L::MASK_OFF + rb * L::MROWP + 15;
        x_stride = L::AREG; hx_rs = L::ROWP; mx_rs = L::MROWP;
      }
    } else {
      if(E.xr) {
        h_x = L::XW_OFF + L::TH * 16 + (R * w) * 16 + (B.wE % L::CH) * L::ESZ;
        m_x = L::XW_OFF + L::NA * L::XWA + L::TH * 16 + (R * w) * 16 + B.wE % 16;
        x_stride = L::XWA; hx_rs = 16; mx_rs = 16;
      } else {
        h_x = rb * L::ROWP + (L::CH + AS_W) * L::ESZ;
        m_x = L::MASK_OFF + rb * L::MROWP + 16 + AS_W;
        x_stride = L::AREG; hx_rs = L::ROWP; mx_rs = L::MROWP;
      }
    }
    const int o_own = L::OWN_OFF + (R * w) * L::OWNB + col * L::ESZ;
    /* carried from plane to plane, per own row: the previous plane's q,
     * its stencil sum without the top term, its mask word and its
     * epilogue inputs */
    T qp[R][4], Pp[R][4], r0p[R][4], r1p[R][4];
    unsigned mp[R];
#pragma unroll
    for(int r = 0; r < R; r++) {
      mp[r] = 0;
#pragma unroll
      for(int v = 0; v < 4; v++) qp[r][v] = Pp[r][v] = r0p[r][v] = r1p[r][v] = (T)0.;
    }
    /* the stage of load L0 + a and its barrier phase, advanced per plane
     * (no 64-bit division in the loop) */
    int buf = (int)(L0 % L::NS);
    uint32_t par = (uint32_t)((L0 / L::NS) & 1);
    for(int a = 0; a < cnt; a++) {
      const int pl = k0 - 1 + a;
      const uint8_t *st = sm + buf * L::STAGE;
      if(!as_wait(as_saddr(&bars[buf]), par)) bad = 1;
      const bool full = pl >= k0 && pl < k1;
      T qk[R][4], qS[4], qN[4], Pk[R][4], r0k[R][4], r1k[R][4];
      T xq[R];
      unsigned mk[R];
#pragma unroll
      for(int r = 0; r < R; r++) { mk[r] = 0; xq[r] = (T)0.; }
      if(nv > 0) {
#pragma unroll
        for(int r = 0; r < R; r++) {
          if(r < nv) {
            mk[r] = *reinterpret_cast<const unsigned *>(st + m_own + r * L::MROWP);
            if(full)
              as_own4<T, PASS>(st + h_own + r * L::ROWP, mk[r], st + o_own + r * L::OWNB,
                tab.dinv, S, lin(B, i0 + col, jw + r, pl), A, qk[r], r0k[r], r1k[r], red);
            else
              as_q4<T, PASS>(st + h_own + r * L::ROWP, mk[r], tab.dinv, S, qk[r]);
          }
        }
        if(full) {
          as_q4<T, PASS>(st + h_s, *reinterpret_cast<const unsigned *>(st + m_s),
            tab.dinv, S, qS);
          as_q4<T, PASS>(st + h_n, *reinterpret_cast<const unsigned *>(st + m_n),
            tab.dinv, S, qN);
          if(tx == 0 || tx == 31) {
#pragma unroll
            for(int r = 0; r < R; r++)
              if(r < nv)
                xq[r] = as_q1<T, PASS>(st + h_x + r * hx_rs, x_stride,
                  st[m_x + r * mx_rs], tab.dinv, S);
          }
        }
      }
      /* release the stage: the last of the warps to finish reading it
       * refills it with the plane NS ahead (no block-wide barrier, so
       * warps drift apart by up to the stage depth) */
      __syncwarp();
      if(tx == 0) {
        uint32_t old = as_release(as_saddr(&rel[buf]));
        if(old % (uint32_t)NW == (uint32_t)(NW - 1) && a + L::NS < cnt)
          as_issue<T, PASS>(B, A, M, sbase + buf * L::STAGE, as_saddr(&bars[buf]),
            i0, j0, mapz(B, pl + L::NS), E);
      }
      if(nv > 0) {
        if(full) {
          /* this plane's stencil up to its top term, while its south,
           * north and x-halo q are at hand */
#pragma unroll
          for(int r = 0; r < R; r++) {
            if(r < nv) {
              T lft = __shfl_up_sync(0xffffffffu, qk[r][3], 1);
              T rgt = __shfl_down_sync(0xffffffffu, qk[r][0], 1);
              if(tx == 0) lft = xq[r];
              if(tx == 31) rgt = xq[r];
              const bool nin = r + 1 < R && r + 1 < nv;
#pragma unroll
              for(int v = 0; v < 4; v++) {
                unsigned mv = mbyte(mk[r], v);
                T qW = v > 0 ? qk[r][v - 1] : lft;
                T qE = v < 3 ? qk[r][v + 1] : rgt;
                T qs = r > 0 ? qk[r > 0 ? r - 1 : 0][v] : qS[v];
                T qn = nin ? qk[r + 1 < R ? r + 1 : r][v] : qN[v];
                Pk[r][v] = as_apply_lo<T>(mv, tab.diag[mv], wx, wy, qp[r][v], qs, qW,
                  qk[r][v], qE, qn, wz);
              }
            }
          }
        }
        if(a >= 2) {
          /* the previous plane completed by its top term */
          const int k = pl - 1;
#pragma unroll
          for(int r = 0; r < R; r++) {
            if(r < nv) {
              T Aq[4];
#pragma unroll
              for(int v = 0; v < 4; v++)
                Aq[v] = as_apply_hi<T>(mbyte(mp[r], v), wz, Pp[r][v], qp[r][v], qk[r][v]);
              const long long ge = lin(B, i0 + col, jw + r, k);
              if constexpr(PASS == 0) {
                as_st4<T>(A.w2 + ge, Aq);
                as_dot4<T>(red[0], r0p[r], Aq);
              } else if constexpr(PASS == 1) {
                as_st4<T>(A.w1 + ge, Aq);
                as_dot4<T>(red[0], Aq, r0p[r]);
                as_dot4<T>(red[1], Aq, Aq);
                as_dot4<T>(red[3], r1p[r], r0p[r]);
                as_dot4<T>(red[4], r1p[r], Aq);
              } else if constexpr(PASS == 3) {
                /* y = A p and (A p, p), as epi_c1 */
                as_st4<T>(A.w1 + ge, Aq);
                as_dot4<T>(red[0], Aq, r0p[r]);
              } else {
                /* outer residual r = b - A x in FP64, stored rounded to FP32 */
                T rr[4];
#pragma unroll
                for(int v = 0; v < 4; v++) rr[v] = r0p[r][v] - Aq[v];
                *reinterpret_cast<float4 *>(A.rf + ge) =
                  make_float4((float)rr[0], (float)rr[1], (float)rr[2], (float)rr[3]);
                as_dot4<T>(red[0], rr, rr);
                as_sum4<T>(red[2], rr);
              }
            }
          }
        }
      }
#pragma unroll
      for(int r = 0; r < R; r++) {
#pragma unroll
        for(int v = 0; v < 4; v++) {
          qp[r][v] = qk[r][v]; Pp[r][v] = Pk[r][v];
          r0p[r][v] = r0k[r][v]; r1p[r][v] = r1k[r][v];
        }
        mp[r] = mk[r];
      }
      if(++buf == L::NS) { buf = 0; par ^= 1u; }
    }
    nload = L0 + cnt;
    u0 += k1 - k0;
    __syncthreads();
  }
  if(__syncthreads_or(bad)) {
    /* a stage never completed: let whatever is still landing finish
     * before the block's shared memory is released */
    if(nload > 0)
      for(int b = 0; b < L::NS; b++) {
        long long last = nload - 1 - ((nload - 1 - b) % L::NS + L::NS) % L::NS;
        if(last >= 0) as_wait(as_saddr(&bars[b]), (uint32_t)((last / L::NS) & 1));
      }
    if(tid == 0) atomicOr(&s->pad, 1);
  }
  /* the pass's reductions and scalar updates, as k_bicgA / k_bicgB /
   * k_outer_resid / k_cg1 */
  if constexpr(PASS == 3) {
    double r1[1] = {red[0]};
    if(bbb_grid_partial<1>(r1, A.partials, &s->ticket, sh)) {
      bbb_grid_finish_sum<1>(r1, A.partials, &s->ticket, sh);
      if(tid == 0) {
        s->alpha = s->rho / r1[0];
        s->first = 0;
        if(((volatile bbb_kry *)s)->pad) { s->status = BBB_ERR_CUDA; s->done = 1; }
      }
    }
  } else if constexpr(PASS == 2) {
    double r3[3] = {red[0], red[1], red[2]};
    if(bbb_grid_partial<3>(r3, A.partials, &s->ticket, sh)) {
      bbb_grid_finish_sum<3>(r3, A.partials, &s->ticket, sh);
      if(tid == 0) {
        bbb_kry *si = A.si;
        double rn = sqrt(r3[0]);
        s->rnorm = rn;
        s->sumx = r3[1];
        s->converged = (rn <= s->tol);
        s->s_conv = 0;
        if(!isfinite(rn)) { s->status = BBB_ERR_NONFINITE; s->done = 1; }
        if(s->converged || s->iter >= s->maxit) s->done = 1;
        if(((volatile bbb_kry *)s)->pad) { s->status = BBB_ERR_CUDA; s->done = 1; }
        double mean = A.project ? r3[2] / (double)A.n : 0.;
        si->sumx = mean;                 /* subtracted by the inner set-up */
        double need = rn > 0. ? 0.5 * s->tol / rn : 1.;
        si->tol = fmax(A.itol, need) * rn;
        si->maxit = A.imaxit;
        si->done = s->done;
        if(s->done) {
          /* no inner sweep follows: it reports no iterations or passes */
          si->iter = 0; si->first = 1; si->s_conv = 0;
        }
      }
    }
  } else if constexpr(PASS == 0) {
    double r4[4] = {red[0], red[1], red[2], red[3]};
    if(bbb_grid_partial<4>(r4, A.partials, &s->ticket, sh)) {
      bbb_grid_finish_sum<4>(r4, A.partials, &s->ticket, sh);
      if(tid == 0) {
        int sconv = s->s_conv;
        if(!S.first) {
          s->sumx = r4[3];
          if(!sconv) s->iter += 1;
        }
        double rn = sconv ? s->rnorm : sqrt(r4[1]);
        s->rnorm = rn;
        s->rho = r4[2];
        s->rhv = r4[0];
        s->alpha = r4[2] / r4[0];
        s->first = 0;
        s->converged = sconv || (rn <= s->tol);
        if(!isfinite(rn)) { s->status = BBB_ERR_NONFINITE; s->done = 1; }
        if(s->converged || s->iter >= s->maxit) s->done = 1;
        if(s->keep && !(rn <= 1e3 * s->rstart)) { s->status = -1; s->done = 1; }
        if(((volatile bbb_kry *)s)->pad) { s->status = BBB_ERR_CUDA; s->done = 1; }
      }
    }
  } else {
    if(bbb_grid_partial<5>(red, A.partials, &s->ticket, sh)) {
      bbb_grid_finish_sum<5>(red, A.partials, &s->ticket, sh);
      if(tid == 0) {
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
          s->beta = (rho_new / s->rho) * (S.alpha / omega);
        }
        if(((volatile bbb_kry *)s)->pad) { s->status = BBB_ERR_CUDA; s->done = 1; }
      }
    }
  }
}

#endif
