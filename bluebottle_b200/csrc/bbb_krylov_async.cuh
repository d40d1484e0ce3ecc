/* bbb_krylov_async.cuh -- the two BiCGSTAB passes with their inputs staged
 * by asynchronous bulk copies (included by bbb_krylov.cu, which defines
 * boxc, opc, optab, op_apply, mapx/y/z, lin, ldv/stv and the reductions).
 *
 * Same arithmetic as k_bicgA / k_bicgB, for rows of a multiple of 128
 * cells.  A block owns a 128 x 8 tile and marches along z; for every plane
 * it needs, one warp issues cp.async.bulk copies of whole 128-cell row
 * segments (plus the 16-byte chunks holding the x-halo cells) of each
 * input array into a shared-memory stage, and the stage's mbarrier
 * completes when all bytes have landed.  Three stages rotate, so two
 * planes are in flight while the block computes the third: the memory
 * system sees long bulk transfers independent of the threads' registers,
 * instead of one load round per plane per thread.  The compute reads the
 * stage exactly as the register version reads global memory.
 *
 * Stage layout (bytes; T the element type, CH = 16 / sizeof(T) cells per
 * 16-byte chunk, W = 128):
 *   halo arrays (pass A: s, t, p, v; pass B: r, v), 10 rows each (tile rows
 *     j0-1 .. j0+8), a row = [CH cells left of the tile | W cells | CH cells
 *     right], the side chunks filled for the 8 tile rows only;
 *   mask, 10 rows of [16 | 128 | 16] bytes;
 *   own arrays (pass A: x, rh; pass B: rh), 8 rows of W cells.
 * Waits on the stage barriers are bounded; a wait that runs out marks the
 * solve failed (status BBB_ERR_CUDA through the scalars) and the kernel
 * carries on without reading stale data past its bounds. */
#ifndef BBB_KRYLOV_ASYNC_CUH
#define BBB_KRYLOV_ASYNC_CUH

#define AS_W 128
#define AS_NS 3
#define AS_THREADS 256

template <typename T, int PASS>
struct as_layout {
  static constexpr int CH = 16 / (int)sizeof(T);
  static constexpr int NA = PASS == 0 ? 4 : 2;        /* halo arrays  */
  static constexpr int NO = PASS == 0 ? 2 : 1;        /* own arrays   */
  static constexpr int ROWB = (AS_W + 2 * CH) * (int)sizeof(T);
  static constexpr int MROWB = 160;
  static constexpr int OWNB = AS_W * (int)sizeof(T);
  static constexpr int HALO_OFF = 0;
  static constexpr int MASK_OFF = NA * 10 * ROWB;
  static constexpr int OWN_OFF = MASK_OFF + 10 * MROWB;
  static constexpr int STAGE = OWN_OFF + NO * 8 * OWNB;
  /* bytes one stage receives */
  static constexpr int TXB = NA * (10 * AS_W * (int)sizeof(T) + 16 * 16)
    + (10 * 128 + 16 * 16) + NO * 8 * OWNB;
  static constexpr int NCOPY = NA * 26 + 26 + NO * 8;
  static constexpr int RING_OFF = AS_NS * STAGE;
  static constexpr int RING = 3 * 10 * AS_W * (int)sizeof(T);
  static constexpr int HWE_OFF = RING_OFF + RING;
  static constexpr int HWE = 2 * 3 * 8 * (int)sizeof(T);
  static constexpr int TAB_OFF = HWE_OFF + HWE;
  static constexpr int TAB = 2 * 128 * (int)sizeof(T);
  static constexpr int BAR_OFF = (TAB_OFF + TAB + 15) / 16 * 16;
  static constexpr int SH_OFF = BAR_OFF + AS_NS * 8;
  static constexpr int SMEM = SH_OFF + 32 * 5 * 8 + 16;
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

__device__ __forceinline__ void as_copy(uint32_t dst, const void *src,
  uint32_t bytes, uint32_t bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
               " [%0], [%1], %2, [%3];"
               :: "r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}

/* bounded wait for the phase of parity `par`; false when the limit ran out */
__device__ __forceinline__ bool as_wait(uint32_t bar, uint32_t par)
{
  for(int it = 0; it < (1 << 21); it++) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(ok) : "r"(bar), "r"(par) : "memory");
    if(ok) return true;
  }
  return false;
}

__device__ __forceinline__ void as_fence_proxy(void)
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

/* the global arrays of one pass */
template <typename T>
struct as_args {
  const uint8_t *mask;
  const T *h[4];          /* halo arrays                                 */
  const T *o[2];          /* own arrays (pass A: x, rh; pass B: rh)      */
  T *w0, *w1, *w2;        /* pass A: r, p_new, v_new; pass B: s, t       */
  T *x;                   /* pass A: x, updated in place                 */
  bbb_kry *s;
  double *partials;
};

/* Issue the bulk copies of plane gk of tile (i0, j0) into stage `st`
 * (warp 0; lane 0 arms the barrier with the stage's byte count first). */
template <typename T, int PASS>
__device__ __forceinline__ void as_issue(const boxc &B, const as_args<T> &A,
  uint8_t *st, uint32_t bar, int i0, int j0, int gk)
{
  typedef as_layout<T, PASS> L;
  int lane = threadIdx.x & 31;
  if(lane == 0) as_expect(bar, (uint32_t)L::TXB);
  __syncwarp();
  int gxl = mapx(B, i0 - 1), gxr = mapx(B, i0 + AS_W);
  int cl = gxl / L::CH * L::CH, cr = gxr / L::CH * L::CH;
  int ml = gxl / 16 * 16, mr = gxr / 16 * 16;
  uint32_t sbase = as_saddr(st);
  for(int c = lane; c < L::NCOPY; c += 32) {
    int grp, q;
    if(c < L::NA * 26) { grp = c / 26; q = c % 26; }
    else if(c < L::NA * 26 + 26) { grp = L::NA; q = c - L::NA * 26; }
    else { grp = L::NA + 1 + (c - L::NA * 26 - 26) / 8; q = (c - L::NA * 26 - 26) % 8; }
    if(grp < L::NA) {                      /* halo array */
      const T *src = A.h[grp];
      uint32_t d = sbase + L::HALO_OFF + grp * 10 * L::ROWB;
      if(q < 10) {
        int gj = mapy(B, j0 - 1 + q);
        as_copy(d + q * L::ROWB + L::CH * (int)sizeof(T), src + lin(B, i0, gj, gk),
          AS_W * sizeof(T), bar);
      } else {
        int r = 1 + (q - 10) / 2, side = (q - 10) % 2;
        int gj = mapy(B, j0 - 1 + r);
        if(side == 0)
          as_copy(d + r * L::ROWB, src + lin(B, cl, gj, gk), 16, bar);
        else
          as_copy(d + r * L::ROWB + (L::CH + AS_W) * (int)sizeof(T),
            src + lin(B, cr, gj, gk), 16, bar);
      }
    } else if(grp == L::NA) {              /* mask */
      uint32_t d = sbase + L::MASK_OFF;
      if(q < 10) {
        int gj = mapy(B, j0 - 1 + q);
        as_copy(d + q * L::MROWB + 16, A.mask + lin(B, i0, gj, gk), 128, bar);
      } else {
        int r = 1 + (q - 10) / 2, side = (q - 10) % 2;
        int gj = mapy(B, j0 - 1 + r);
        if(side == 0)
          as_copy(d + r * L::MROWB, A.mask + lin(B, ml, gj, gk), 16, bar);
        else
          as_copy(d + r * L::MROWB + 144, A.mask + lin(B, mr, gj, gk), 16, bar);
      }
    } else {                               /* own array rows 1..8 */
      int b = grp - L::NA - 1, r = 1 + q;
      int gj = mapy(B, j0 - 1 + r);
      as_copy(sbase + L::OWN_OFF + b * 8 * L::OWNB + q * L::OWNB,
        A.o[b] + lin(B, i0, gj, gk), L::OWNB, bar);
    }
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

/* pass scalars, read once per kernel */
struct as_scal {
  double alpha, omega, beta, bo;
  int first;
};

/* The stencil input q at 4 consecutive cells of staged row `row` starting
 * at tile column `col`, and, for cells the block owns (`own`), the pass's
 * pointwise work: stores to global index gc and sums into red.  raw0/raw1
 * carry what the epilogue needs (pass A: rh; pass B: s, rh). */
template <typename T, int PASS>
__device__ __forceinline__ void as_cell4(const uint8_t *st, int row, int col,
  const T *dinv, const as_scal &S, bool own, long long gc,
  const as_args<T> &A, T (&q)[4], T (&raw0)[4], T (&raw1)[4], unsigned &mw,
  double (&red)[5])
{
  typedef as_layout<T, PASS> L;
  const int ho = (L::CH + col) * (int)sizeof(T);
  mw = *reinterpret_cast<const unsigned *>(st + L::MASK_OFF + row * L::MROWB + 16 + col);
  if constexpr(PASS == 0) {
    T ss[4], rr[4], pn[4];
    as_ld4<T>(st + L::HALO_OFF + 0 * 10 * L::ROWB + row * L::ROWB + ho, ss);
    T al = (T)S.alpha, om = (T)S.omega, be = (T)S.beta, bo = (T)S.bo;
    if(S.first) {
#pragma unroll
      for(int a = 0; a < 4; a++) { rr[a] = ss[a]; pn[a] = rr[a]; }
    } else {
      T tt[4], pp[4], vv[4];
      as_ld4<T>(st + L::HALO_OFF + 1 * 10 * L::ROWB + row * L::ROWB + ho, tt);
      as_ld4<T>(st + L::HALO_OFF + 2 * 10 * L::ROWB + row * L::ROWB + ho, pp);
      as_ld4<T>(st + L::HALO_OFF + 3 * 10 * L::ROWB + row * L::ROWB + ho, vv);
#pragma unroll
      for(int a = 0; a < 4; a++) {
        rr[a] = ss[a] - om * tt[a];
        pn[a] = rr[a] + be * pp[a] + bo * vv[a];
      }
      if(own) {
        T xx[4];
        as_ld4<T>(st + L::OWN_OFF + (row - 1) * L::OWNB + col * (int)sizeof(T), xx);
#pragma unroll
        for(int a = 0; a < 4; a++) {
          T di = dinv[mbyte(mw, a)];
          xx[a] = xx[a] + al * (di * pp[a]) + om * (di * ss[a]);
          red[3] += (double)xx[a];
        }
        as_st4<T>(A.x + gc, xx);
      }
    }
#pragma unroll
    for(int a = 0; a < 4; a++) q[a] = dinv[mbyte(mw, a)] * pn[a];
    if(own) {
      as_ld4<T>(st + L::OWN_OFF + 8 * L::OWNB + (row - 1) * L::OWNB
        + col * (int)sizeof(T), raw0);
#pragma unroll
      for(int a = 0; a < 4; a++) {
        red[1] += (double)rr[a] * (double)rr[a];
        red[2] += (double)raw0[a] * (double)rr[a];
      }
      as_st4<T>(A.w0 + gc, rr);
      as_st4<T>(A.w1 + gc, pn);
    } else {
#pragma unroll
      for(int a = 0; a < 4; a++) raw0[a] = (T)0.;
    }
  } else {
    T rr[4], vv[4];
    as_ld4<T>(st + L::HALO_OFF + 0 * 10 * L::ROWB + row * L::ROWB + ho, rr);
    as_ld4<T>(st + L::HALO_OFF + 1 * 10 * L::ROWB + row * L::ROWB + ho, vv);
    T al = (T)S.alpha;
#pragma unroll
    for(int a = 0; a < 4; a++) {
      raw0[a] = rr[a] - al * vv[a];
      q[a] = dinv[mbyte(mw, a)] * raw0[a];
    }
    if(own) {
      as_ld4<T>(st + L::OWN_OFF + (row - 1) * L::OWNB + col * (int)sizeof(T), raw1);
#pragma unroll
      for(int a = 0; a < 4; a++) red[2] += (double)raw0[a] * (double)raw0[a];
      as_st4<T>(A.w0 + gc, raw0);
    } else {
#pragma unroll
      for(int a = 0; a < 4; a++) raw1[a] = (T)0.;
    }
  }
}

/* q at one x-halo cell: staged row `row`, byte offset `boff` inside the
 * halo-array row and `moff` inside the mask row */
template <typename T, int PASS>
__device__ __forceinline__ T as_cell1(const uint8_t *st, int row, int boff,
  int moff, const T *dinv, const as_scal &S)
{
  typedef as_layout<T, PASS> L;
  unsigned m = st[L::MASK_OFF + row * L::MROWB + moff];
  const uint8_t *h = st + L::HALO_OFF + row * L::ROWB + boff;
  if constexpr(PASS == 0) {
    T ss = *reinterpret_cast<const T *>(h);
    T pn;
    if(S.first) pn = ss;
    else {
      T tt = *reinterpret_cast<const T *>(h + 1 * 10 * L::ROWB);
      T pp = *reinterpret_cast<const T *>(h + 2 * 10 * L::ROWB);
      T vv = *reinterpret_cast<const T *>(h + 3 * 10 * L::ROWB);
      T rr = ss - (T)S.omega * tt;
      pn = rr + (T)S.beta * pp + (T)S.bo * vv;
    }
    return dinv[m] * pn;
  } else {
    T rr = *reinterpret_cast<const T *>(h);
    T vv = *reinterpret_cast<const T *>(h + 1 * 10 * L::ROWB);
    T ss = rr - (T)S.alpha * vv;
    return dinv[m] * ss;
  }
}

/* One BiCGSTAB pass (PASS 0: pass A, 1: pass B) over this block's units,
 * 256 threads = 8 warps, warp w owning tile row w, lane l cells 4l..4l+3.
 * Per plane: wait for the stage, produce q (own cells, halo rows by warps
 * 0-1, halo columns by 16 threads of warp 2), one barrier, re-arm the
 * stage with the plane three ahead, then the stencil and epilogue of the
 * plane below. */
template <typename T, int PASS>
__global__ void __launch_bounds__(AS_THREADS) k_bicg_async(boxc B, opc O,
  as_args<T> A)
{
  typedef as_layout<T, PASS> L;
  bbb_kry *s = A.s;
  if(((volatile bbb_kry *)s)->done) return;
  extern __shared__ __align__(128) uint8_t as_sm[];
  T (*ring)[10][AS_W] = reinterpret_cast<T (*)[10][AS_W]>(as_sm + L::RING_OFF);
  T *hwe = reinterpret_cast<T *>(as_sm + L::HWE_OFF);   /* [side][slot][row] */
  optab<T> &tab = *reinterpret_cast<optab<T> *>(as_sm + L::TAB_OFF);
  uint64_t *bars = reinterpret_cast<uint64_t *>(as_sm + L::BAR_OFF);
  double *sh = reinterpret_cast<double *>(as_sm + L::SH_OFF);
  int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  if(tid == 0) {
    for(int b = 0; b < AS_NS; b++) as_bar_init(as_saddr(&bars[b]));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  optab_fill<T>(tab, O);                  /* ends with a barrier */
  as_scal S;
  S.alpha = s->alpha; S.omega = s->omega; S.beta = s->beta;
  S.bo = -S.beta * S.omega; S.first = s->first;
  double red[5] = {0., 0., 0., 0., 0.};
  int bad = 0;
  long long nload = 0;
  long long bxl = blockIdx.x;
  long long u0 = bxl * B.q + (bxl < B.r ? bxl : B.r);
  long long u1 = u0 + B.q + (bxl < B.r ? 1 : 0);
  int gxl = 0, gxr = 0;
  while(u0 < u1) {
    long long tile = u0 / B.nz;
    int k0 = (int)(u0 - tile * B.nz);
    long long left_ = u1 - u0;
    int k1 = left_ < (long long)(B.nz - k0) ? k0 + (int)left_ : B.nz;
    int i0 = (int)(tile % B.tiles_x) * AS_W, j0 = (int)(tile / B.tiles_x) * 8;
    int j = j0 + ty;
    bool valid = j < B.ny;
    gxl = mapx(B, i0 - 1); gxr = mapx(B, i0 + AS_W);
    int cnt = k1 - k0 + 2;
    long long L0 = nload;
    if(ty == 0)
      for(int a = 0; a < AS_NS && a < cnt; a++) {
        int b = (int)((L0 + a) % AS_NS);
        as_issue<T, PASS>(B, A, as_sm + b * L::STAGE, as_saddr(&bars[b]), i0, j0,
          mapz(B, k0 - 1 + a));
      }
    T qm[4], qc[4], qn[4], r0c[4], r1c[4], r0n[4], r1n[4];
    unsigned mc = 0, mn = 0;
#pragma unroll
    for(int v = 0; v < 4; v++) {
      qm[v] = qc[v] = qn[v] = (T)0.;
      r0c[v] = r1c[v] = r0n[v] = r1n[v] = (T)0.;
    }
    for(int a = 0; a < cnt; a++) {
      int pl = k0 - 1 + a;
      long long Ld = L0 + a;
      int buf = (int)(Ld % AS_NS);
      uint32_t par = (uint32_t)((Ld / AS_NS) & 1);
      uint8_t *st = as_sm + buf * L::STAGE;
      if(!as_wait(as_saddr(&bars[buf]), par)) bad = 1;
      bool full = pl >= k0 && pl < k1;
      bool own = valid && full;
      long long gc = own ? lin(B, i0 + tx * 4, j, pl) : 0;
      as_cell4<T, PASS>(st, ty + 1, tx * 4, tab.dinv, S, own, gc, A, qn, r0n,
        r1n, mn, red);
      if(full) {
        int slot = (pl - k0) % 3;
        as_st4<T>(&ring[slot][ty + 1][tx * 4], qn);
        if(tid < 64) {
          int hr = tid < 32 ? 0 : 9;
          T hq[4], d0[4], d1[4];
          unsigned hm;
          as_cell4<T, PASS>(st, hr, (tid & 31) * 4, tab.dinv, S, false, 0, A,
            hq, d0, d1, hm, red);
          as_st4<T>(&ring[slot][hr][(tid & 31) * 4], hq);
        } else if(tid < 80) {
          int side = tid < 72 ? 0 : 1, r = 1 + ((tid - 64) & 7);
          int boff, moff;
          if(side == 0) {
            boff = (gxl - gxl / L::CH * L::CH) * (int)sizeof(T);
            moff = gxl - gxl / 16 * 16;
          } else {
            boff = (L::CH + AS_W + (gxr - gxr / L::CH * L::CH)) * (int)sizeof(T);
            moff = 144 + (gxr - gxr / 16 * 16);
          }
          hwe[(side * 3 + slot) * 8 + (r - 1)] =
            as_cell1<T, PASS>(st, r, boff, moff, tab.dinv, S);
        }
      }
      as_fence_proxy();
      __syncthreads();
      if(a + AS_NS < cnt && ty == 0)
        as_issue<T, PASS>(B, A, st, as_saddr(&bars[buf]), i0, j0,
          mapz(B, pl + AS_NS));
      if(a >= 2) {
        int k = pl - 1, sl = (k - k0) % 3;
        T lft = __shfl_up_sync(0xffffffffu, qc[3], 1);
        T rgt = __shfl_down_sync(0xffffffffu, qc[0], 1);
        if(tx == 0) lft = hwe[(0 * 3 + sl) * 8 + ty];
        if(tx == 31) rgt = hwe[(1 * 3 + sl) * 8 + ty];
        if(valid) {
          T Sv[4], Nv[4], Aq[4];
          as_ld4<T>(reinterpret_cast<const uint8_t *>(&ring[sl][ty][tx * 4]), Sv);
          as_ld4<T>(reinterpret_cast<const uint8_t *>(&ring[sl][ty + 2][tx * 4]), Nv);
#pragma unroll
          for(int v = 0; v < 4; v++) {
            unsigned mv = mbyte(mc, v);
            T qW = v > 0 ? qc[v - 1] : lft;
            T qE = v < 3 ? qc[v + 1] : rgt;
            Aq[v] = op_apply<T>(mv, O, tab.diag[mv], qm[v], Sv[v], qW, qc[v], qE,
              Nv[v], qn[v]);
          }
          long long ge = lin(B, i0 + tx * 4, j, k);
          if constexpr(PASS == 0) {
            as_st4<T>(A.w2 + ge, Aq);
#pragma unroll
            for(int v = 0; v < 4; v++) red[0] += (double)r0c[v] * (double)Aq[v];
          } else {
            as_st4<T>(A.w1 + ge, Aq);
#pragma unroll
            for(int v = 0; v < 4; v++) {
              red[0] += (double)Aq[v] * (double)r0c[v];
              red[1] += (double)Aq[v] * (double)Aq[v];
              red[3] += (double)r1c[v] * (double)r0c[v];
              red[4] += (double)r1c[v] * (double)Aq[v];
            }
          }
        }
      }
#pragma unroll
      for(int v = 0; v < 4; v++) {
        qm[v] = qc[v]; qc[v] = qn[v]; r0c[v] = r0n[v]; r1c[v] = r1n[v];
      }
      mc = mn;
    }
    nload = L0 + cnt;
    u0 += k1 - k0;
    __syncthreads();
  }
  if(__syncthreads_or(bad)) {
    /* a stage never completed: let whatever is still landing finish
     * before the block's shared memory is released */
    for(int b = 0; b < AS_NS; b++) {
      long long last = nload - 1 - ((nload - 1 - b) % AS_NS + AS_NS) % AS_NS;
      if(last >= 0) as_wait(as_saddr(&bars[b]), (uint32_t)((last / AS_NS) & 1));
    }
    if(tid == 0) atomicOr(&s->pad, 1);
  }
  /* the pass's reductions and scalar updates, as k_bicgA / k_bicgB */
  if constexpr(PASS == 0) {
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
        s->alpha = r4[2] / r4[0];
        s->first = 0;
        s->converged = sconv || (rn <= s->tol);
        if(!isfinite(rn)) { s->status = BBB_ERR_NONFINITE; s->done = 1; }
        if(s->converged || s->iter >= s->maxit) s->done = 1;
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
        int sconv = (sn <= s->tol);
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
