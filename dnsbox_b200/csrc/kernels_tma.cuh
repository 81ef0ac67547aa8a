// Tensor-core split-precision strided pass with TMA-staged tiles
// (DNSBOX_TC_SPLIT, FP32 data), used by the right-hand side.
//
// A length-N transform along the strided axis (N = 64 N2) is split by
// decimation in time, n = 64 n2 + n1, k = k2 + N2 k1:
//   X[k2 + N2 k1] = sum_n1 W64^(n1 k1) [ W_N^(n1 k2) sum_n2 W_N2^(n2 k2) x[64 n2 + n1] ]
// Stage A (FP32 SIMT) forms the bracket: an N2-point DFT over n2 and the
// twiddle, for every (n1, column).  Stage B is the 64-point DFT over n1 as a
// dense real contraction on the tensor cores:
//   D[m][j'] = sum_n1 A[m][n1] B[n1][j'],
// A = the DFT-64 matrix with the rows of its real and imaginary parts
// interleaved (m = 2 k1 + {0, 1}), B = the stage-A values of the tile's 64
// pencils j = k2 TCW + c with their real and imaginary parts interleaved
// (j' = 2 j + {0, 1}).  Then Re Y[k1][j] = D[2k1][2j] - D[2k1+1][2j+1] and
// Im Y[k1][j] = D[2k1][2j+1] + D[2k1+1][2j], combined in FP32 by the lane
// pair that holds TMEM rows 2 k1 and 2 k1 + 1, and Y[k1][(k2, c)] is output
// row k2 + N2 k1 of column c: the drain stores straight from registers.
//
// Operands are f16 hi + lo splits (hi = rn(x), lo = rn(x - hi)); each column
// of a tile is scaled by the power of two that brings its largest |Re|, |Im|
// into [0.5, 1) first and unscaled exactly in the drain.  Each accumulator
// takes Al Xh, Ah Xl, then Ah Xh (the tensor core adds into its accumulator
// with truncation relative to the largest addend, so the small correction
// products go first); the lo x lo term (2^-22 relative) is dropped.  The real
// and imaginary parts of X sit in different accumulator columns, so each
// accumulation chain is one 64-term real dot product.
//
// Data movement: one thread issues the tile's input loads as TMA boxes of 8
// rows (only the rows the pass keeps, when pruning) into a staging tile that
// completes on an mbarrier; the next tile's loads are in flight while the
// current one is processed (two staging buffers, or one staging buffer per
// input for two-input jobs).  The B operands are double buffered and written
// in the MN-major 128-byte-swizzle layout, so the MMAs of one tile run while
// stage A of the next proceeds, and the accumulators (two 128-column TMEM
// regions) are drained one tile behind.  One persistent CTA of 512 threads
// per SM.  Every wait is bounded: a wait that gives up sets the status flag,
// the copies and MMAs in flight are waited for (again bounded), TMEM is freed
// and the kernel returns.
#pragma once

#include <cuda.h>

#include "kernels_tc.cuh"

namespace dnsbox {

template <int N> struct TmaPlan {
  static constexpr bool on = N == 128 || N == 256 || N == 512;
  static constexpr int N2 = on ? N / 64 : 1;
  static constexpr int TCW = 64 / N2;            // kx columns per tile
  static constexpr int G = on ? 8 / N2 : 1;      // columns per stage-A item: G * N2 = 8 values a thread
  static constexpr int SPC = TCW + 2;            // staging row pitch (complex): the tile and a one-column shift
  static constexpr int STAGE = N * SPC * 8;      // bytes of one staged input tile
  static constexpr int THREADS = 512;            // 64 n1 x 8 column groups
  static constexpr int A_PART = 128 * 64 * 2;    // f16 128 x 64 operand
  static constexpr int B_PART = 64 * 128 * 2;    // f16 64 (K) x 128 (MN) operand
  static constexpr int TMEM_COLS = 256;          // two 128-column accumulators
  static constexpr int SMEM = 1024 + 2 * A_PART + 4 * B_PART + 2 * STAGE;
};

constexpr int kTmaMaxBoxes = 64;   // boxes per staged tile (N / 8 at most)

struct TmaJob {
  const float2 *in1, *in2;   // field pointers (the merged Nyquist column is read through them)
  float2 *out;
  float a1, b1, a2, b2;      // multipliers a + i b k
  int ks1, ks2;              // k: 0 kx of the column, 1 the row index's, 2 the tile's other-axis index's
  int slot1, slot2;          // slot coordinate of in1 / in2 in the tensor map (in2: -1 none)
};

struct TmaArgs {
  // the inputs as a 5D float tensor; y pass over the padded workspace:
  // (x = 2 kx + re/im, row y, other z, box, slot), z pass over the state:
  // (x = 2 (y nxh + kx) + re/im within a plane, row z, box, component, 1)
  CUtensorMap map;
  TmaJob job[6];
  const float2 *tw;          // exp(-2 pi i j / N), j < N
  long long rowstride;       // input strides (complex elements), for the merged Nyquist column
  long long otherstride, bstride;
  long long rso, oso, bso;   // output strides (complex elements, even)
  int njobs;
  int plane;                 // 1: z pass over the state (x = (other, kx) within a plane), 0: y pass over rows
  int in_pitch;              // plane mode: complex elements per (other) row of a plane
  int two;                   // 1: a job has two inputs (one staging buffer per input)
  int ncols, nx, n_other;
  float alpha_row, alpha_x, alpha_other;
  int nbox;                  // boxes per staged input tile
  int box_rows;              // rows per box (8, 16, 32 or 64; the tensor map's box height)
  unsigned short box_row[kTmaMaxBoxes];
  AxisKeep kcol, koth, krin, krout;
  int ntx_lo, nyq_tile;
  int total;                 // work items: boxes x tiles x jobs
  FastDiv per_box, njobs_d, ntxd;
};

namespace tma {
__device__ __forceinline__ void expect_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(mbar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void load5(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3, int c4,
                                      uint64_t *mbar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5, %6}], [%7];" ::"r"(tc::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(tc::smem_u32(mbar))
      : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// shared-memory descriptor of an MN-major operand in the 128-byte swizzle
// layout (version 1, layout type 2, base offset 0: atoms 1024-byte aligned)
__device__ __forceinline__ uint64_t desc_sw128(const void *p, uint32_t lbo, uint32_t sbo) {
  return tc::smem_desc(p, lbo, sbo) | ((uint64_t)2 << 61);
}
// byte offset of f16 element (k, m) of a 64 (K) x 128 (MN) MN-major operand in
// the 128-byte swizzle layout: 64-element MN atoms 8 KB apart (LBO), 8-row K
// groups 1 KB apart (SBO), 16-byte chunk index XOR row within the group
__device__ __forceinline__ int b_offset(int k, int m) {
  const int chunk = ((m & 63) >> 3) ^ (k & 7);
  return (m >> 6) * 8192 + (k >> 3) * 1024 + (k & 7) * 128 + chunk * 16 + (m & 7) * 2;
}
}  // namespace tma

constexpr int kTmaWaitLimit = 1 << 22;

// Work item w -> (job, column origin, other-axis index, box).
struct TmaItem {
  int job, kx0, other, box;
};
template <int TCW> __device__ __forceinline__ TmaItem tma_item(const TmaArgs &a, unsigned w) {
  TmaItem it;
  const unsigned box = a.per_box.div(w);
  const unsigned rw = w - box * a.per_box.d;
  const unsigned tile = a.njobs_d.div(rw);
  it.job = (int)(rw - tile * a.njobs_d.d);
  const int o = (int)a.ntxd.div(tile);
  const int kt = (int)(tile - (unsigned)o * a.ntxd.d);
  it.other = a.koth.map(o);
  it.kx0 = (a.ntx_lo == 0 || kt < a.ntx_lo ? kt : a.nyq_tile) * TCW;
  it.box = (int)box;
  return it;
}

// Half-axis index held by tile column kx0 + c (the merged Nyquist slot maps
// to kcol.n / 2).
__device__ __forceinline__ int tma_col(const TmaArgs &a, int kx) {
  return (a.nyq_tile < 0 && kx == a.kcol.a) ? (a.kcol.n >> 1) : kx;
}

template <int N, bool INV>
__global__ void __launch_bounds__(TmaPlan<N>::THREADS, 1)
    k_strided_tma(const __grid_constant__ TmaArgs a, const __half *__restrict__ Adft, int *status) {
  using C = float2;
  using PL = TmaPlan<N>;
  constexpr int N2 = PL::N2, TCW = PL::TCW, G = PL::G, SPC = PL::SPC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  unsigned char *sAh = base;                        // K-major, no swizzle
  unsigned char *sAl = base + PL::A_PART;
  unsigned char *sB = base + 2 * PL::A_PART;        // [buffer][hi, lo], 1024-byte aligned
  unsigned char *stg = sB + 4 * PL::B_PART;         // staging: [2][N][SPC] complex
  __shared__ __align__(8) uint64_t full[2], mmab[2];
  __shared__ uint32_t taddr_s;
  __shared__ int abort_s;
  __shared__ unsigned pm[3][TCW];      // per-column max |Re|, |Im| bits, rotating over tiles
  __shared__ float krow[N];            // wavenumber of each row index along the transformed axis
  __shared__ C tws[(N2 - 1) * 64];     // W_N^(n1 k2), k2 = 1 .. N2-1
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  for (int i = t; i < (N2 - 1) * 64; i += PL::THREADS) tws[i] = a.tw[(i / 64 + 1) * (i % 64)];
  for (int n = t; n < N; n += PL::THREADS) krow[n] = (float)k_full(n, N, a.alpha_row);
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(Adft);
    uint4 *dst = reinterpret_cast<uint4 *>(sAh);
    for (int i = t; i < 2 * PL::A_PART / 16; i += PL::THREADS) dst[i] = src[i];
  }
  if (t < 3 * TCW) pm[t / TCW][t % TCW] = 0u;
  if (warp == 0) {
    tc::tmem_alloc(&taddr_s, PL::TMEM_COLS);
    tc::tmem_relinquish();
  }
  if (t == 0) {
    tc::mbar_init(&full[0], 1);
    tc::mbar_init(&full[1], 1);
    tc::mbar_init(&mmab[0], 1);
    tc::mbar_init(&mmab[1], 1);
    tma::fence_mbar_init();
    abort_s = 0;
  }
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = taddr_s;
  constexpr uint32_t idesc = (1u << 4) | (1u << 16) | ((uint32_t)(128 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
  const int NST = a.two ? 1 : 2;      // staging buffers in rotation
  const unsigned nb = gridDim.x;
  const int my_n = (int)blockIdx.x < a.total ? (a.total - (int)blockIdx.x + (int)nb - 1) / (int)nb : 0;
  const uint32_t box_bytes = (uint32_t)a.box_rows * SPC * 8;

  // tile i of this CTA: loads into staging buffer s, issued by the lanes of
  // warp 0 (one box each, after lane 0 has armed the barrier)
  auto issue_loads = [&](int i, int s) {
    const TmaItem it = tma_item<TCW>(a, blockIdx.x + (unsigned)i * nb);
    const TmaJob &J = a.job[it.job];
    const int nin = J.slot2 >= 0 ? 2 : 1;
    if (lane == 0) tma::expect_tx(&full[s], (uint32_t)(nin * a.nbox) * box_bytes);
    __syncwarp();
    const int off = it.other * a.in_pitch + it.kx0;   // plane mode: column index within the plane
    const int x = a.plane ? 2 * (off - (off & 1)) : 2 * it.kx0;   // 16-byte aligned start
    for (int k = lane; k < nin * a.nbox; k += 32) {
      const int q = k >= a.nbox ? 1 : 0, b = k - q * a.nbox;
      const int slot = q ? J.slot2 : J.slot1;
      unsigned char *dst = stg + (size_t)(s + q) * PL::STAGE + (size_t)a.box_row[b] * SPC * 8;
      const int r0 = a.box_row[b];
      if (a.plane) tma::load5(dst, &a.map, x, r0, it.box, slot, 0, &full[s]);
      else tma::load5(dst, &a.map, x, r0, it.other, it.box, slot, &full[s]);
    }
  };

  // stage-A item of this thread: n1 (four per warp, chosen so that the
  // warp's operand stores fall in distinct bank groups) and column group cg
  const int cg = lane & 7, jq = lane >> 3;
  constexpr int D1 = G >= 2 ? 1 : 2;
  const int n1 = 8 * (warp >> 1) + (jq & 1) * D1 + 4 * (jq >> 1) + (warp & 1) * (D1 == 1 ? 2 : 1);
  const int c0 = cg * G;

  if (warp == 0)
    for (int i = 0; i < NST && i < my_n; ++i) issue_loads(i, i);
  // Tile k of this CTA uses staging buffer k % NST with mbarrier parity
  // (k / NST) & 1 and accumulator k & 1 with parity (k >> 1) & 1.  Thread 0
  // counts the tiles whose loads it issued and whose loads / MMAs it saw
  // complete, for the bounded clean-up after an abort.
  int loads_issued = NST < my_n ? NST : my_n, loads_seen = 0, mma_issued = 0, mma_seen = 0;
  TmaItem prev{};
  bool aborted = false;
  for (int i = 0; i <= my_n; ++i) {
    const int bb = i & 1;
    if (i < my_n) {
      const int s = NST == 2 ? (i & 1) : 0;
      const TmaItem it = tma_item<TCW>(a, blockIdx.x + (unsigned)i * nb);
      const TmaJob &J = a.job[it.job];
      // ---- wait for the staged tile (every thread polls, bounded)
      if (tc::mbar_wait_bounded(&full[s], (uint32_t)(i / NST) & 1u, kTmaWaitLimit)) ++loads_seen;
      else abort_s = 1;
      // ---- stage A: multipliers, N2-point DFT, twiddle, column maxima
      const C *st1 = reinterpret_cast<const C *>(stg + (size_t)s * PL::STAGE);
      const C *st2 = reinterpret_cast<const C *>(stg + (size_t)(s + 1) * PL::STAGE);
      const int shift = a.plane ? ((it.other * a.in_pitch + it.kx0) & 1) : 0;
      const float koth = a.n_other ? (float)k_full(it.other, a.n_other, a.alpha_other) : 0.f;
      C z[G][N2];
      float cmax[G];
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const int c = c0 + g;
        const int kx = tma_col(a, it.kx0 + c);
        const bool valid = kx < a.ncols && a.kcol.keep(kx);
        const bool slotcol = kx != it.kx0 + c;   // merged Nyquist column: read from global memory
        const float kcol = (float)k_half(kx, a.nx, a.alpha_x);
        const float kc1 = J.ks1 == 2 ? koth : kcol, kc2 = J.ks2 == 2 ? koth : kcol;
        const long long gbase = (long long)it.box * a.bstride + (long long)it.other * a.otherstride + kx;
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) {
          const int n = 64 * n2 + n1;
          const bool ok = valid && a.krin.keep(n);
          C v = mkc<C>(0.f, 0.f);
          if (ok) {
            v = slotcol ? J.in1[gbase + (long long)n * a.rowstride] : st1[n * SPC + c + shift];
            if (!(J.a1 == 1.f && J.b1 == 0.f)) {
              const float bk = J.b1 * (J.ks1 == 1 ? krow[n] : kc1);
              v = mkc<C>(v.x * J.a1 - v.y * bk, v.y * J.a1 + v.x * bk);
            }
            if (J.slot2 >= 0) {
              const C w2 = slotcol ? J.in2[gbase + (long long)n * a.rowstride] : st2[n * SPC + c + shift];
              const float bk = J.b2 * (J.ks2 == 1 ? krow[n] : kc2);
              v = mkc<C>(v.x + (w2.x * J.a2 - w2.y * bk), v.y + (w2.y * J.a2 + w2.x * bk));
            }
          }
          z[g][n2] = v;
        }
        dft<N2, C, INV>(z[g]);
        float m = fmaxf(fabsf(z[g][0].x), fabsf(z[g][0].y));
#pragma unroll
        for (int k2 = 1; k2 < N2; ++k2) {
          const C tw = tws[(k2 - 1) * 64 + n1];
          z[g][k2] = INV ? cmulc(z[g][k2], tw) : cmul(z[g][k2], tw);
          m = fmaxf(m, fmaxf(fabsf(z[g][k2].x), fabsf(z[g][k2].y)));
        }
        // the warp's four n1 of this column group are lanes cg + 8 jq
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 8));
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 16));
        cmax[g] = m;
      }
      unsigned *pmi = pm[i % 3];
      if (jq == 0)
#pragma unroll
        for (int g = 0; g < G; ++g) atomicMax(&pmi[c0 + g], __float_as_uint(cmax[g]));
      __syncthreads();   // #1: column maxima complete
      if (abort_s) {
        aborted = true;
        break;
      }
      if (t < TCW) pm[(i + 1) % 3][t] = 0u;   // used by tile i - 2, drained in the previous iteration
      // ---- scale, split into f16 hi + lo, store the B operands
      unsigned char *Bh = sB + (size_t)bb * 2 * PL::B_PART, *Bl = Bh + PL::B_PART;
      float sc[G];
#pragma unroll
      for (int g = 0; g < G; ++g) sc[g] = __int_as_float((127 - tc_exp(pmi[c0 + g])) << 23);   // 2^-e
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        __align__(16) __half2 hv[G], lv[G];
#pragma unroll
        for (int g = 0; g < G; ++g) {
          const float2 x = make_float2(z[g][k2].x * sc[g], z[g][k2].y * sc[g]);
          hv[g] = __float22half2_rn(x);
          const float2 hb = __half22float2(hv[g]);
          lv[g] = __float22half2_rn(make_float2(x.x - hb.x, x.y - hb.y));
        }
        const int off = tma::b_offset(n1, 2 * (k2 * TCW + c0));
        if constexpr (G == 4) {
          *reinterpret_cast<uint4 *>(Bh + off) = *reinterpret_cast<const uint4 *>(hv);
          *reinterpret_cast<uint4 *>(Bl + off) = *reinterpret_cast<const uint4 *>(lv);
        } else if constexpr (G == 2) {
          *reinterpret_cast<uint2 *>(Bh + off) = *reinterpret_cast<const uint2 *>(hv);
          *reinterpret_cast<uint2 *>(Bl + off) = *reinterpret_cast<const uint2 *>(lv);
        } else {
          *reinterpret_cast<__half2 *>(Bh + off) = hv[0];
          *reinterpret_cast<__half2 *>(Bl + off) = lv[0];
        }
      }
      tc::fence_proxy_async();
      tc::fence_before_sync();
      __syncthreads();   // #2: operands written, staging buffer s consumed
      if (warp == 0) {
        tc::fence_after_sync();
        if (loads_issued < my_n) {
          issue_loads(loads_issued, NST == 2 ? (loads_issued & 1) : 0);
          ++loads_issued;
        }
      }
      if (t == 0) {
        // 3 x 4 MMAs (K = 16 each) into accumulator bb: Al Bh, Ah Bl, then Ah Bh
        constexpr uint32_t lboA = (128 / 8) * 128, sboA = 128, lboB = 8192, sboB = 1024;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const unsigned char *A = p == 0 ? sAl : sAh;
          const unsigned char *B = p == 1 ? Bl : Bh;
#pragma unroll
          for (int ks = 0; ks < 4; ++ks)
            tc::mma_f16(taddr + 128u * bb, tc::smem_desc(A + 2 * ks * lboA, lboA, sboA),
                        tma::desc_sw128(B + 2 * ks * sboB, lboB, sboB), idesc, (p | ks) ? 1u : 0u);
        }
        tc::mma_commit(&mmab[bb]);
        ++mma_issued;
      }
    }
    // ---- drain the previous tile
    if (i >= 1) {
      const int pb = (i - 1) & 1;
      if (t == 0) {
        if (tc::mbar_wait_bounded(&mmab[pb], (uint32_t)((i - 1) >> 1) & 1u, kTmaWaitLimit)) ++mma_seen;
        else abort_s = 1;
      }
      tc::fence_before_sync();
      __syncthreads();   // #3
      tc::fence_after_sync();
      if (abort_s) {
        aborted = true;
        break;
      }
      const TmaItem it = prev;
      const TmaJob &J = a.job[it.job];
      const int q = warp & 3, g4 = warp >> 2;
      const uint32_t ta = taddr + ((uint32_t)(32 * q) << 16) + 128u * pb + 32u * g4;
      float v[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]),
            "=f"(v[8]), "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15]),
            "=f"(v[16]), "=f"(v[17]), "=f"(v[18]), "=f"(v[19]), "=f"(v[20]), "=f"(v[21]), "=f"(v[22]), "=f"(v[23]),
            "=f"(v[24]), "=f"(v[25]), "=f"(v[26]), "=f"(v[27]), "=f"(v[28]), "=f"(v[29]), "=f"(v[30]), "=f"(v[31])
          : "r"(ta)
          : "memory");
      tc::tmem_ld_wait();
      const bool odd = lane & 1;
      const int k1 = 16 * q + (lane >> 1);
      const unsigned *pmd = pm[(i - 1) % 3];
      float w[16];
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) {
        const float tpart = __shfl_xor_sync(0xffffffffu, v[2 * jj + 1], 1);
        const int c = (16 * g4 + jj) % TCW;
        const float us = __int_as_float((127 + tc_exp(pmd[c])) << 23);   // 2^e
        w[jj] = (odd ? tpart + v[2 * jj] : v[2 * jj] - tpart) * us;
      }
      // even lane: pencils 0..7 (re own, im from the odd lane); odd lane: 8..15
      float r[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) r[k] = __shfl_xor_sync(0xffffffffu, odd ? w[k] : w[8 + k], 1);
      const int jbase = 16 * g4 + (odd ? 8 : 0);
      const long long obase = (long long)it.box * a.bso + (long long)it.other * a.oso;
#pragma unroll
      for (int k = 0; k < 8; k += 2) {
        const int j = jbase + k;
        const int k2 = j / TCW, c = j % TCW;   // c even: the pair (c, c + 1) shares the output row
        const int row = k2 + N2 * k1;
        if (!a.krout.keep(row)) continue;
        const C y0 = odd ? mkc<C>(r[k], w[8 + k]) : mkc<C>(w[k], r[k]);
        const C y1 = odd ? mkc<C>(r[k + 1], w[9 + k]) : mkc<C>(w[k + 1], r[k + 1]);
        const int kx0c = it.kx0 + c;
        const int kxa = tma_col(a, kx0c), kxb = tma_col(a, kx0c + 1);
        const bool va = kxa < a.ncols && a.kcol.keep(kxa), vb = kxb < a.ncols && a.kcol.keep(kxb);
        C *orow = J.out + obase + (long long)row * a.rso;
        if (va && vb && kxa == kx0c && kxb == kx0c + 1) {
          *reinterpret_cast<float4 *>(orow + kx0c) = make_float4(y0.x, y0.y, y1.x, y1.y);
        } else {
          if (va) orow[kxa] = y0;
          if (vb) orow[kxb] = y1;
        }
      }
    }
    if (i < my_n) prev = tma_item<TCW>(a, blockIdx.x + (unsigned)i * nb);
  }
  if (aborted && t == 0) {
    // wait (bounded) for the copies and MMAs still in flight before TMEM is freed
    for (int k = loads_seen; k < loads_issued; ++k)
      tc::mbar_wait_bounded(&full[NST == 2 ? (k & 1) : 0], (uint32_t)(k / NST) & 1u, kTmaWaitLimit);
    for (int k = mma_seen; k < mma_issued; ++k)
      tc::mbar_wait_bounded(&mmab[k & 1], (uint32_t)(k >> 1) & 1u, kTmaWaitLimit);
    atomicExch(status, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, PL::TMEM_COLS);
}

}  // namespace dnsbox
