// Tensor-core split-precision strided pass (DNSBOX_TC_SPLIT), FP32 data.
//
// A length-N transform along the strided axis is split as N = 64 * N2
// (Cooley-Tukey, n = N2 n1 + n2, k = k1 + 64 k2):
//   stage 1  y[n2][k1] = sum_n1 F[k1][n1] x[N2 n1 + n2],  F = W64^(k1 n1)     tensor cores
//   stage 2  X[k1 + 64 k2] = sum_n2 W_N2^(n2 k2) (W_N^(n2 k1) y[n2][k1])      FP32 SIMT
// A tile is TCW = 64 / N2 consecutive kx columns, i.e. 64 "pencils" (n2, c) of
// 64 inputs each.  With A the rows of F's real and imaginary parts interleaved
// (128 x 64: row 2k = Fr[k], row 2k + 1 = Fi[k]) and the pencils' real and
// imaginary parts Xr, Xi (64 x 64 each, rows = pencils j = n2 TCW + c)
// stage 1 is two dense real contractions
//   DR = A Xr^T,  DI = A Xi^T   (128 x 64 each),
//   Re y[k] = DR[2k] - DI[2k + 1],  Im y[k] = DR[2k + 1] + DI[2k],
// so each pair of adjacent TMEM lanes combines with one warp shuffle.
// Every pencil is first scaled by the power of two that brings its largest
// |Re|, |Im| into [0.5, 1), which keeps both f16 parts in range and is undone
// exactly on the way out.  A and X are split into f16 hi + lo parts and each
// of DR, DI = Al Xh + Ah Xl + Ah Xh is accumulated in FP32 in tensor memory by
// 12 tcgen05.mma of K = 16 issued by one thread (the lo x lo term, 2^-22
// relative, is dropped).  The tensor core adds into its accumulator with
// truncation relative to the largest addend, so the small correction
// products are issued first, while the accumulator is still small; with the
// two accumulators combined in round-to-nearest FP32 afterwards one pass has
// close to the error of the FP32 SIMT transform.
//
// Resources per CTA: A hi + lo for the direction (32 KB, resident for the
// whole persistent launch), X hi + lo (32 KB; the FP32 tile D of the combined
// accumulators reuses it once the MMAs have completed, XOR-swizzled so that
// the TMEM drain and the stage-2 reads are free of bank conflicts), 128 TMEM
// columns and 512 threads, plus a 32 KB ring into which the next tile's first
// input is copied asynchronously.  Two CTAs share an SM, and each fetches its
// next tile while the current one is split, multiplied, drained and stored,
// so the loads, MMAs and stores of different tiles overlap.
#pragma once

#include <cuda_fp16.h>

#include "kernels.cuh"
#include "tc.cuh"

namespace dnsbox {

template <int N> struct TcPlan {
  static constexpr bool on = N == 128 || N == 256 || N == 512 || N == 1024;
  static constexpr int N2 = on ? N / 64 : 1;
  static constexpr int TCW = 64 / N2;              // kx columns per tile
  static constexpr int LG_R = N2 == 2 ? 0 : N2 == 4 ? 1 : N2 == 8 ? 2 : 3;   // log2(32 / TCW)
  static constexpr int A_PART = 128 * 64 * 2;      // bytes of one f16 128 x 64 A operand
  static constexpr int B_PART = 64 * 128 * 2;      // bytes of one f16 64 x 128 X operand (Re | Im)
  static constexpr int TILE = 64 * 64 * 8;         // bytes of one FP32 complex tile (N x TCW)
  static constexpr int SMEM = 2 * A_PART + 2 * B_PART + TILE;
  static constexpr int THREADS = 512;              // 8-row runs of one pencil: RUNS per thread
  static constexpr int RUNS = 512 / THREADS;
  static constexpr int CTAS_PER_SM = 2;
  static constexpr int TMEM_COLS = 128;            // DR, DI: 64 columns each
};

// Bytes of the host-built DFT-64 operand block: forward hi, forward lo,
// inverse hi, inverse lo, each a 128 x 64 f16 K-major operand (rows Fr[k],
// Fi[k] interleaved).
constexpr int kTcDftBytes = 4 * 128 * 64 * 2;
constexpr int kTcWaitLimit = 1 << 22;   // polls of the MMA completion barrier (each may suspend)

// Column swizzle of row r of the D tile: a bijection of r mod 32 that sends
// the 2^LG_R consecutive rows read by one warp in stage 2 to distinct
// TCW-wide bank groups.  Imaginary rows additionally flip bit 4 - LG_R, which
// is constant over the 16 rows one warp drains, so the drain's real and
// imaginary writes also fall in distinct banks.
template <int LG_R> __device__ __forceinline__ int tc_swz(int r) {
  return ((r & ((1 << LG_R) - 1)) << (5 - LG_R)) | ((r >> LG_R) & ((32 >> LG_R) - 1));
}

// Exponent e of a pencil maximum m = f 2^e, f in [0.5, 1), from its bits (a
// zero pencil gives 0), clamped to [-126, 126] so that 2^-e and 2^e are both
// normal floats.
__device__ __forceinline__ int tc_exp(unsigned bits) {
  const int e = bits ? (int)((bits >> 23) & 255u) - 126 : 0;
  return e < -126 ? -126 : (e > 126 ? 126 : e);
}

// Unsigned 32-bit division by an invariant divisor d >= 1 with one high
// multiply (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, the round-up variant): with l = ceil(log2 d)
// and m = floor(2^32 (2^l - d) / d) + 1, t = mulhi(m, n) gives
// n / d = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0) for every 32-bit n.
struct FastDiv {
  unsigned d, m;
  int s1, s2;
  __host__ void init(unsigned dd) {
    d = dd;
    int l = 0;
    while ((1ull << l) < dd) ++l;
    m = (unsigned)(((1ull << 32) * ((1ull << l) - dd)) / dd + 1);
    s1 = l < 1 ? l : 1;
    s2 = l > 1 ? l - 1 : 0;
  }
  __host__ __device__ __forceinline__ unsigned div(unsigned n) const {
#ifdef __CUDA_ARCH__
    const unsigned t = __umulhi(m, n);
#else
    const unsigned t = (unsigned)(((unsigned long long)m * n) >> 32);
#endif
    return (t + ((n - t) >> s1)) >> s2;
  }
};

struct TcArgs {
  int ntx;          // kept tiles across the kx columns (all when not pruning)
  int nother;       // kept indices of the other axis
  int total;        // work items: boxes x tiles x jobs (< 2^31)
  FastDiv per_box;  // njobs * ntx * nother
  FastDiv njobs;
  FastDiv ntxd;     // ntx
};

// 8-byte asynchronous global -> shared copy; zero-fills when !valid.
__device__ __forceinline__ void cp_async8(void *dst, const void *src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(tc::smem_u32(dst)), "l"(src),
               "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Work item w -> (job, base offset, column origin, other-axis index).
struct TcItem {
  int job, kx0, other;
  long long base0, base0o;   // input and output offsets of the tile origin
};
template <int TCW>
__device__ __forceinline__ TcItem tc_item(const StridedArgs<float> &a, const TcArgs &g, unsigned w) {
  const unsigned box = g.per_box.div(w);
  const unsigned rw = w - box * g.per_box.d;
  const unsigned tile = g.njobs.div(rw);
  TcItem it;
  it.job = (int)(rw - tile * g.njobs.d);
  const int o = (int)g.ntxd.div(tile);
  const int kt = (int)(tile - (unsigned)o * g.ntxd.d);
  it.other = a.koth.map(o);
  it.kx0 = (a.ntx_lo == 0 || kt < a.ntx_lo ? kt : a.nyq_tile) * TCW;
  it.base0 = (long long)box * a.bstride + (long long)it.other * a.otherstride + it.kx0;
  it.base0o = (long long)box * out_bstride(a) + (long long)it.other * out_otherstride(a) + it.kx0;
  return it;
}

template <int N, bool INV>
__global__ void __launch_bounds__(TcPlan<N>::THREADS, TcPlan<N>::CTAS_PER_SM)
    k_strided_tc(const __grid_constant__ StridedArgs<float> a, const TcArgs g, const __half *__restrict__ Adft,
                 int *status) {
  using C = float2;
  using PL = TcPlan<N>;
  constexpr int N2 = PL::N2, TCW = PL::TCW, LG_R = PL::LG_R, NT = PL::THREADS, RUNS = PL::RUNS;
  constexpr int XIM = 1 << (4 - LG_R);   // swizzle bit flipped for imaginary rows
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *sAh = smem_raw;
  unsigned char *sAl = smem_raw + PL::A_PART;
  unsigned char *sBh = smem_raw + 2 * PL::A_PART;
  unsigned char *sBl = sBh + PL::B_PART;
  float *sD = reinterpret_cast<float *>(sBh);   // 128 x 64: rows Re y[k1], Im y[k1]; aliases X
  C *ring = reinterpret_cast<C *>(sBh + 2 * PL::B_PART);   // next tile's first input, per-thread slots
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t taddr_s;
  __shared__ unsigned pmax_s[2][64];   // per-pencil max |Re|, |Im| bits, alternating tiles
  __shared__ int abort_s;
  __shared__ float usc[64];            // this tile's per-pencil unscale factors 2^e
  __shared__ float krow[N];            // wavenumber of each row index along the transformed axis
  __shared__ StridedJob<float> sjob[6];   // the job table (read with a per-tile index)
  __shared__ C tws[(N2 - 1) * 64];        // stage-2 twiddles W_N^(m2 k1), m2 = 1 .. N2-1
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  if (t < a.njobs) sjob[t] = a.job[t];
  for (int i = t; i < (N2 - 1) * 64; i += NT) tws[i] = a.tw[(i / 64 + 1) * (i % 64)];
  for (int n = t; n < N; n += NT) krow[n] = (float)k_full(n, N, a.alpha_row);
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(Adft);
    uint4 *dst = reinterpret_cast<uint4 *>(sAh);
    for (int i = t; i < 2 * PL::A_PART / 16; i += NT) dst[i] = src[i];
  }
  if (warp == 0) {
    tc::tmem_alloc(&taddr_s, PL::TMEM_COLS);
    tc::tmem_relinquish();
  }
  if (t == 0) {
    tc::mbar_init(&mbar, 1);
    abort_s = 0;
  }
  if (t < 128) pmax_s[t >> 6][t & 63] = 0u;
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = taddr_s;
  constexpr uint32_t idesc = tc::idesc_f16_f32(128, 64);
  uint32_t phase = 0;
  int slot = 0;
  // Thread t owns, for h < RUNS, the 8-row run u = t + NT h of the tile:
  // rows n = N2 (8q + i) + n2 (i < 8) of column c, with c = u % TCW,
  // n2 = (u / TCW) % N2, q = u / 64, i.e. pencil j = u % 64.  The next tile's
  // first input is copied asynchronously into the thread's own 8 RUNS ring
  // slots (slot (8 h + i) * NT + t, consecutive across a warp; no barrier guards
  // the ring) and its second input, if any, is loaded into registers, both
  // while the current tile is processed.
  C y[RUNS][8];
  TcItem nxt;   // decoded work item of the tile being fetched
  // Row offsets within one field fit in 32 bits (the launcher checks
  // N * rowstride < 2^31); the 64-bit part is the per-tile base.
  const int rs = (int)a.rowstride, rso = (int)out_rowstride(a);
  // Kept-row masks, fixed per thread for the whole launch: bit 8 h + i for
  // input row N2 (8 q + i) + n2 of run h, bit N2 r + k2 for output row
  // k1 + 64 k2 of stage-2 item r.
  constexpr int R2 = (64 * TCW + NT - 1) / NT;   // stage-2 items per thread
  unsigned inmask = 0, outmask = 0;
#pragma unroll
  for (int h = 0; h < RUNS; ++h) {
    const int u = t + NT * h;
    const int n2 = (u / TCW) % N2, q = u / 64;
#pragma unroll
    for (int i = 0; i < 8; ++i) inmask |= (a.krin.keep(N2 * (8 * q + i) + n2) ? 1u : 0u) << (8 * h + i);
  }
  // With half as many stage-2 items as threads (N2 = 16), a lane pair shares
  // item t / 2: lane parity s takes the inputs m2 = 2 r + s and the outputs
  // k2 = 8 s + k (bit k of outmask).
  constexpr bool PAIR = 2 * 64 * TCW == NT;
  if constexpr (PAIR) {
    const int k1 = (t >> 1) / TCW, sp = t & 1;
#pragma unroll
    for (int k = 0; k < 8; ++k) outmask |= (a.krout.keep(k1 + 64 * (8 * sp + k)) ? 1u : 0u) << k;
  } else {
#pragma unroll
    for (int r = 0; r < R2; ++r) {
      const int k1 = (t + NT * r) / TCW;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) outmask |= (a.krout.keep(k1 + 64 * k2) ? 1u : 0u) << (N2 * r + k2);
    }
  }
  auto fetch = [&](unsigned w) {
    nxt = tc_item<TCW>(a, g, w);
    const TcItem &it = nxt;
    const StridedJob<float> &J = sjob[it.job];
#pragma unroll
    for (int h = 0; h < RUNS; ++h) {
      const int u = t + NT * h;
      const int c = u % TCW, n2 = (u / TCW) % N2, q = u / 64;
      const int dc = strided_col(a, it.kx0 + c) - it.kx0;   // column offset from the tile origin
      const bool valid = it.kx0 + dc < a.ncols && a.kcol.keep(it.kx0 + dc);
      const int roff = (N2 * 8 * q + n2) * rs;
      const C *src1 = J.in1 + (it.base0 + dc);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const bool vi = valid && ((inmask >> (8 * h + i)) & 1u);
        cp_async8(ring + (8 * h + i) * NT + t, vi ? src1 + (roff + N2 * i * rs) : J.in1, vi);
      }
      if (J.in2) {
        const C *src2 = J.in2 + (it.base0 + dc);
#pragma unroll
        for (int i = 0; i < 8; ++i)
          y[h][i] = (valid && ((inmask >> (8 * h + i)) & 1u)) ? src2[roff + N2 * i * rs] : mkc<C>(0.f, 0.f);
      }
    }
    cp_async_commit();
  };
  if (blockIdx.x < (unsigned)g.total) fetch(blockIdx.x);   // (sjob is visible: init barrier above)
  for (unsigned w = blockIdx.x; w < (unsigned)g.total; w += gridDim.x, slot ^= 1) {
    const TcItem it = nxt;   // decoded by the fetch of this tile
    const StridedJob<float> J = sjob[it.job];   // job fields in registers for the tile
    unsigned *pmax = pmax_s[slot];
    C v[RUNS][8];
    cp_async_wait_all();
#pragma unroll
    for (int h = 0; h < RUNS; ++h)
#pragma unroll
      for (int i = 0; i < 8; ++i) v[h][i] = ring[(8 * h + i) * NT + t];
    // 1. the second input and the job multipliers x (a + i b k), in FP32
    const bool mult1 = !(J.a1 == 1.0 && J.b1 == 0.0);
    if (mult1 || J.in2) {
      const float a1 = (float)J.a1, b1 = (float)J.b1, a2 = (float)J.a2, b2 = (float)J.b2;
      const float koth = a.n_other ? (float)k_full(it.other, a.n_other, a.alpha_other) : 0.f;
#pragma unroll
      for (int h = 0; h < RUNS; ++h) {
        const int u = t + NT * h;
        const int c = u % TCW, n2 = (u / TCW) % N2, q = u / 64;
        const float kcol = (float)k_half(strided_col(a, it.kx0 + c), a.nx, a.alpha_x);
        const float kc1 = J.ks1 == 2 ? koth : kcol, kc2 = J.ks2 == 2 ? koth : kcol;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int n = N2 * (8 * q + i) + n2;
          if (mult1) {
            const float bk = b1 * (J.ks1 == 1 ? krow[n] : kc1);
            v[h][i] = mkc<C>(v[h][i].x * a1 - v[h][i].y * bk, v[h][i].y * a1 + v[h][i].x * bk);
          }
          if (J.in2) {
            const float bk = b2 * (J.ks2 == 1 ? krow[n] : kc2);
            v[h][i] = mkc<C>(v[h][i].x + (y[h][i].x * a2 - y[h][i].y * bk),
                             v[h][i].y + (y[h][i].y * a2 + y[h][i].x * bk));
          }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < RUNS; ++h) {
      float m = 0.f;
#pragma unroll
      for (int i = 0; i < 8; ++i) m = fmaxf(m, fmaxf(fabsf(v[h][i].x), fabsf(v[h][i].y)));
      atomicMax(&pmax[(t + NT * h) % 64], __float_as_uint(m));   // non-negative floats order as unsigned
    }
    __syncthreads();
    if (t < 64) {
      pmax_s[slot ^ 1][t] = 0u;   // for the next tile (its atomics follow the end barrier)
      usc[t] = __int_as_float((127 + tc_exp(pmax[t])) << 23);   // 2^e, read back in stage 2
    }
    // 2. scale, split into f16 hi + lo, 16-byte stores of 8 consecutive K
    //    (K = n1 for the real parts, 64 + n1 for the imaginary parts)
#pragma unroll
    for (int h = 0; h < RUNS; ++h) {
      const int u = t + NT * h;
      const int j = u % 64, q = u / 64;
      const float sc = __int_as_float((127 - tc_exp(pmax[j])) << 23);   // 2^-e
      // packed conversions (two values per instruction): hi = rn(x), lo = rn(x - hi)
      __align__(16) __half2 hr[4], hi[4], lr[4], li[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float2 xr = make_float2(v[h][2 * i].x * sc, v[h][2 * i + 1].x * sc);
        const float2 xi = make_float2(v[h][2 * i].y * sc, v[h][2 * i + 1].y * sc);
        hr[i] = __float22half2_rn(xr);
        hi[i] = __float22half2_rn(xi);
        const float2 br = __half22float2(hr[i]), bi = __half22float2(hi[i]);
        lr[i] = __float22half2_rn(make_float2(xr.x - br.x, xr.y - br.y));
        li[i] = __float22half2_rn(make_float2(xi.x - bi.x, xi.y - bi.y));
      }
      const int ore = tc::kmajor_offset(j, 8 * q, 64), oim = tc::kmajor_offset(j, 64 + 8 * q, 64);
      *reinterpret_cast<uint4 *>(sBh + ore) = *reinterpret_cast<const uint4 *>(hr);
      *reinterpret_cast<uint4 *>(sBh + oim) = *reinterpret_cast<const uint4 *>(hi);
      *reinterpret_cast<uint4 *>(sBl + ore) = *reinterpret_cast<const uint4 *>(lr);
      *reinterpret_cast<uint4 *>(sBl + oim) = *reinterpret_cast<const uint4 *>(li);
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    // 3. DR (TMEM columns 0..63) from the real K half, DI (64..127) from the
    //    imaginary half: Al Xh, Ah Xl, then Ah Xh, four K-steps of 16 each
    if (t == 0) {
      tc::fence_after_sync();
      constexpr uint32_t lboA = (128 / 8) * 128, lboB = (64 / 8) * 128, sbo = 128;
#pragma unroll
      for (int part = 0; part < 2; ++part) {
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const unsigned char *A = p == 0 ? sAl : sAh;
          const unsigned char *B = p == 1 ? sBl : sBh;
#pragma unroll
          for (int ks = 0; ks < 4; ++ks)
            tc::mma_f16(taddr + 64u * part, tc::smem_desc(A + 2 * ks * lboA, lboA, sbo),
                        tc::smem_desc(B + 2 * (4 * part + ks) * lboB, lboB, sbo), idesc, (p | ks) ? 1u : 0u);
        }
      }
      tc::mma_commit(&mbar);
    }
    // the next tile is fetched while the tensor core runs (after the proxy
    // fence above, which would otherwise wait for these copies)
    if (w + gridDim.x < (unsigned)g.total) fetch(w + gridDim.x);
    // one thread polls the MMA completion (the others wait at the barrier,
    // which costs no issue slots or shared-memory accesses)
    if (t == 0 && !tc::mbar_wait_bounded(&mbar, phase, kTcWaitLimit)) abort_s = 1;
    tc::fence_after_sync();
    __syncthreads();
    if (abort_s) break;
    phase ^= 1u;
    // 4. drain: warp w reads TMEM lanes 32 (w % 4) + lane and DCOL columns from
    //    DCOL (w / 4) of DR and DI; lane pair (2k, 2k + 1) forms Re y[k] and Im y[k]
    {
      constexpr int DCOL = 64 / (NT / 128);   // columns per warp
      const int k1 = 16 * (warp & 3) + (lane >> 1);
      const bool odd = lane & 1;
      const int sw = tc_swz<LG_R>(k1) ^ (odd ? XIM : 0);
      float *row = sD + (odd ? 64 + k1 : k1) * 64;
      const uint32_t ta = taddr + ((uint32_t)(32 * (warp & 3)) << 16);
#pragma unroll
      for (int part = 0; part < DCOL / 8; ++part) {
        const int c0 = DCOL * (warp >> 2) + 8 * part;
        float dr[8], di[8];
        tc::tmem_ld8(ta + (uint32_t)c0, dr);
        tc::tmem_ld8(ta + 64u + (uint32_t)c0, di);
        tc::tmem_ld_wait();
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float dip = __shfl_xor_sync(0xffffffffu, di[k], 1);
          row[(c0 + k) ^ sw] = odd ? dr[k] + dip : dr[k] - dip;
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();
    // 5. unscale, twiddle, N2-point DFT, store; item (k1, c), c fastest.
    //    Paired form (N2 = 16), decimation in time: lane s forms the 8-point
    //    DFT of the inputs m2 = 2 r + s, the odd lane multiplies by W16^k, the
    //    pair exchanges them, and X[k] = E[k] + W O[k] (even lane),
    //    X[k + 8] = E[k] - W O[k] (odd lane).
    if constexpr (PAIR) {
      const int item = t >> 1, sp = t & 1;
      const int cc = item % TCW, k1 = item / TCW;
      const int sw = tc_swz<LG_R>(k1), swi = sw ^ XIM;
      C z[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int m2 = 2 * r + sp;
        const int jj = m2 * TCW + cc;
        const float us = usc[jj];
        C yy = mkc<C>(sD[k1 * 64 + (jj ^ sw)] * us, sD[(64 + k1) * 64 + (jj ^ swi)] * us);
        if (m2) {
          const C tw = tws[(m2 - 1) * 64 + k1];
          yy = INV ? cmulc(yy, tw) : cmul(yy, tw);
        }
        z[r] = yy;
      }
      dft<8, C, INV>(z);
      // exp(-2 pi i k / 16), k < 8
      constexpr float kc[8] = {1.f, 0.92387953251128676f, 0.70710678118654752f, 0.38268343236508977f,
                               0.f, -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128676f};
      constexpr float ks[8] = {0.f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128676f,
                               1.f, 0.92387953251128676f, 0.70710678118654752f, 0.38268343236508977f};
      if (sp) {
#pragma unroll
        for (int k = 1; k < 8; ++k) {
          const C w = mkc<C>(kc[k], -ks[k]);
          z[k] = INV ? cmulc(z[k], w) : cmul(z[k], w);
        }
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const C o = mkc<C>(__shfl_xor_sync(0xffffffffu, z[k].x, 1), __shfl_xor_sync(0xffffffffu, z[k].y, 1));
        z[k] = sp ? csub(o, z[k]) : cadd(z[k], o);
      }
      const int dc = strided_col(a, it.kx0 + cc) - it.kx0;
      if (it.kx0 + dc < a.ncols && a.kcol.keep(it.kx0 + dc)) {
        C *out = J.out + (it.base0o + dc);
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if ((outmask >> k) & 1u) out[(k1 + 64 * (8 * sp + k)) * rso] = z[k];
      }
    } else
#pragma unroll
    for (int r = 0; r < R2; ++r) {
      const int idx = t + NT * r;
      if ((64 * TCW) % NT != 0 && idx >= 64 * TCW) break;
      const int cc = idx % TCW, k1 = idx / TCW;
      const int sw = tc_swz<LG_R>(k1), swi = sw ^ XIM;
      C z[N2];
#pragma unroll
      for (int m2 = 0; m2 < N2; ++m2) {
        const int jj = m2 * TCW + cc;
        const float us = usc[jj];
        C yy = mkc<C>(sD[k1 * 64 + (jj ^ sw)] * us, sD[(64 + k1) * 64 + (jj ^ swi)] * us);
        if (m2) {
          const C tw = tws[(m2 - 1) * 64 + k1];
          yy = INV ? cmulc(yy, tw) : cmul(yy, tw);
        }
        z[m2] = yy;
      }
      dft<N2, C, INV>(z);
      const int dc = strided_col(a, it.kx0 + cc) - it.kx0;
      if (it.kx0 + dc < a.ncols && a.kcol.keep(it.kx0 + dc)) {
        C *out = J.out + (it.base0o + dc);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2)
          if ((outmask >> (N2 * r + k2)) & 1u) out[(k1 + 64 * k2) * rso] = z[k2];
      }
    }
    __syncthreads();
  }
  cp_async_wait_all();
  if (abort_s && t == 0) {
    // give the outstanding MMAs a second bounded wait before their TMEM is freed
    tc::mbar_wait_bounded(&mbar, phase, kTcWaitLimit);
    atomicExch(status, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, PL::TMEM_COLS);
}

}  // namespace dnsbox
