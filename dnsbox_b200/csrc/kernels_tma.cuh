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
// Data movement: the lanes of warp 0 issue the tile's input loads as TMA
// boxes (only the rows the pass keeps, when pruning) into a staging tile that
// completes on an mbarrier; the next tile's loads are issued as soon as the
// current tile's stage A has read the staging tile, so they land while its
// DFT, split and MMAs run (a two-input job stages its second input after the
// first).  Two 256-thread CTAs share an SM, each with its own staging tile, B
// operand (MN-major 128-byte swizzle) and 128-column TMEM accumulator, so the
// phases and waits of one overlap the work of the other; a tile's
// accumulator is drained straight to HBM at the start of the next tile's
// split, before the next MMAs are issued.  Per-tile column data (half-axis
// index, wavenumber, unscale factor) is tabulated once in shared memory and
// the thread's kept-row masks and row offsets once per launch.  Every wait is
// bounded (one thread polls each barrier): a wait that gives up sets the
// status flag, the copies and MMAs in flight are waited for (again bounded),
// TMEM is freed and the kernel returns.
#pragma once

#include <cuda.h>

#include "kernels_tc.cuh"

namespace dnsbox {

template <int N> struct TmaPlan {
  static constexpr bool on = N == 128 || N == 256 || N == 512;
  static constexpr int N2 = on ? N / 64 : 1;
  static constexpr int TCW = 64 / N2;            // kx columns per tile
  static constexpr int G = on ? 8 / N2 : 1;      // columns per stage-A item: G * N2 = 8 values
  static constexpr int SPC = TCW + 2;            // staging row pitch (complex): the tile and a one-column shift
  static constexpr int STAGE = N * SPC * 8;      // bytes of the staged input tile
  static constexpr int THREADS = 256;            // 8 warps; 512 stage-A items (64 n1 x 8 column groups), 2 each
  static constexpr int CTAS_PER_SM = 2;
  static constexpr int A_PART = 128 * 64 * 2;    // f16 128 x 64 operand
  static constexpr int B_PART = 64 * 128 * 2;    // f16 64 (K) x 128 (MN) operand
  static constexpr int TMEM_COLS = 128;          // one 128-column accumulator
  static constexpr int SMEM = 1024 + 2 * A_PART + 2 * B_PART + STAGE;
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
__global__ void __launch_bounds__(TmaPlan<N>::THREADS, TmaPlan<N>::CTAS_PER_SM)
    k_strided_tma(const __grid_constant__ TmaArgs a, const __half *__restrict__ Adft, int *status) {
  using C = float2;
  using PL = TmaPlan<N>;
  constexpr int N2 = PL::N2, TCW = PL::TCW, G = PL::G, SPC = PL::SPC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  unsigned char *sAh = base;                        // K-major, no swizzle
  unsigned char *sAl = base + PL::A_PART;
  unsigned char *sBh = base + 2 * PL::A_PART;       // MN-major, 128-byte swizzle, 1024-byte aligned
  unsigned char *sBl = sBh + PL::B_PART;
  const C *stg = reinterpret_cast<const C *>(sBh + 2 * PL::B_PART);   // staging: [N][SPC] complex
  __shared__ __align__(8) uint64_t full, mmab;
  __shared__ uint32_t taddr_s;
  __shared__ int abort_s;
  __shared__ unsigned pm[2][TCW];              // per-column max |Re|, |Im| bits (tile parity)
  __shared__ __align__(16) float usc[2][TCW];  // per-column unscale 2^e (tile parity)
  __shared__ int colkx[2][TCW];                // half-axis index of each tile column, -1 if not kept (tile parity)
  __shared__ float colk[TCW];                  // its wavenumber
  __shared__ float krow[N];                    // wavenumber of each row index along the transformed axis
  __shared__ C tws[(N2 - 1) * 64];             // W_N^(n1 k2), k2 = 1 .. N2-1
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  for (int i = t; i < (N2 - 1) * 64; i += PL::THREADS) tws[i] = a.tw[(i / 64 + 1) * (i % 64)];
  for (int n = t; n < N; n += PL::THREADS) krow[n] = (float)k_full(n, N, a.alpha_row);
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(Adft);
    uint4 *dst = reinterpret_cast<uint4 *>(sAh);
    for (int i = t; i < 2 * PL::A_PART / 16; i += PL::THREADS) dst[i] = src[i];
  }
  if (t < 2 * TCW) pm[t / TCW][t % TCW] = 0u;
  if (warp == 0) {
    tc::tmem_alloc(&taddr_s, PL::TMEM_COLS);
    tc::tmem_relinquish();
  }
  if (t == 0) {
    tc::mbar_init(&full, 1);
    tc::mbar_init(&mmab, 1);
    tma::fence_mbar_init();
    abort_s = 0;
  }
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = taddr_s;
  constexpr uint32_t idesc = (1u << 4) | (1u << 16) | ((uint32_t)(128 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
  const unsigned nb = gridDim.x;
  const int my_n = (int)blockIdx.x < a.total ? (a.total - (int)blockIdx.x + (int)nb - 1) / (int)nb : 0;
  const uint32_t box_bytes = (uint32_t)a.box_rows * SPC * 8;

  // one staged input of tile i (input q: 0 in1, 1 in2), issued by the lanes
  // of warp 0 (one box each) after lane 0 has armed the barrier
  auto issue_load = [&](int i, int q) {
    const TmaItem it = tma_item<TCW>(a, blockIdx.x + (unsigned)i * nb);
    const int slot = q ? a.job[it.job].slot2 : a.job[it.job].slot1;
    if (lane == 0) tma::expect_tx(&full, (uint32_t)a.nbox * box_bytes);
    __syncwarp();
    const int off = it.other * a.in_pitch + it.kx0;   // plane mode: column index within the plane
    const int x = a.plane ? 2 * (off - (off & 1)) : 2 * it.kx0;   // 16-byte aligned start
    for (int b = lane; b < a.nbox; b += 32) {
      const int r0 = a.box_row[b];
      unsigned char *dst = const_cast<unsigned char *>(reinterpret_cast<const unsigned char *>(stg)) +
                           (size_t)r0 * SPC * 8;
      if (a.plane) tma::load5(dst, &a.map, x, r0, it.box, slot, 0, &full);
      else tma::load5(dst, &a.map, x, r0, it.other, it.box, slot, &full);
    }
  };

  // Stage-A items of this thread: item h covers n1(h) (four per warp, chosen
  // so that a warp's operand stores fall in distinct bank groups) and the G
  // columns c0 .. c0 + G - 1.
  const int cg = lane & 7, jq = lane >> 3;
  constexpr int D1 = G >= 2 ? 1 : 2;
  int n1s[2];
  unsigned rin = 0;   // kept input rows: bit h N2 + n2 for row 64 n2 + n1(h)
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int vw = warp + 8 * h;
    n1s[h] = 8 * (vw >> 1) + (jq & 1) * D1 + 4 * (jq >> 1) + (vw & 1) * (D1 == 1 ? 2 : 1);
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) rin |= (a.krin.keep(64 * n2 + n1s[h]) ? 1u : 0u) << (h * N2 + n2);
  }
  const int c0 = cg * G;
  // Drain: warp w reads TMEM lanes 32 (w % 4) + lane (k1 = 16 (w % 4) + lane / 2)
  // and the two 32-column blocks 64 (w / 4) .. + 63 (pencils 32 (w / 4) .. + 31).
  const int q4 = warp & 3;
  const bool odd = lane & 1;
  const int k1 = 16 * q4 + (lane >> 1);
  unsigned rout = 0;  // kept output rows: bit 4 sb + k / 2 for pair k of sub-block sb
  int roff[8];        // their row offsets (complex elements)
#pragma unroll
  for (int sb = 0; sb < 2; ++sb)
#pragma unroll
    for (int k = 0; k < 8; k += 2) {
      const int j = 32 * (warp >> 2) + 16 * sb + (odd ? 8 : 0) + k;
      const int row = j / TCW + N2 * k1;
      rout |= (a.krout.keep(row) ? 1u : 0u) << (4 * sb + k / 2);
      roff[4 * sb + k / 2] = row * (int)a.rso;
    }

  // Tile k uses the staging barrier once per input (parity = running input
  // count & 1) and the MMA barrier once (parity k & 1).  Thread 0 counts the
  // inputs and MMAs issued and seen, for the bounded clean-up after an abort.
  int loads_issued = 0, loads_seen = 0, mma_issued = 0, mma_seen = 0;
  if (warp == 0 && my_n > 0) {
    issue_load(0, 0);
    ++loads_issued;
  }
  TmaItem prev{};
  bool aborted = false;
  auto wait_load = [&]() {   // thread 0
    if (tc::mbar_wait_bounded(&full, (uint32_t)loads_seen & 1u, kTmaWaitLimit)) ++loads_seen;
    else abort_s = 2;   // the status code says which wait gave up: 2 staged copy, 3 MMA
  };
  for (int i = 0; i <= my_n; ++i) {
    const int par = i & 1;
    C z[2][G][N2];   // stage-A values of this thread's items (tile i)
    if (i < my_n) {
      const TmaItem it = tma_item<TCW>(a, blockIdx.x + (unsigned)i * nb);
      const TmaJob J = a.job[it.job];
      const bool two = J.slot2 >= 0;
      // ---- per-tile column table, staging wait
      if (t < TCW) {
        const int kx = tma_col(a, it.kx0 + t);
        const bool ok = kx < a.ncols && a.kcol.keep(kx);
        colkx[par][t] = ok ? kx : -1;
        colk[t] = (float)k_half(kx, a.nx, a.alpha_x);
      }
      if (t == 0) wait_load();
      __syncthreads();   // A: staged input 1 and the column table visible
      if (abort_s) {
        aborted = true;
        break;
      }
      if (t < TCW) pm[par ^ 1][t] = 0u;   // for tile i + 1 (its last reader, tile i - 1's split, is done)
      const int shift = a.plane ? ((it.other * a.in_pitch + it.kx0) & 1) : 0;
      const float koth = a.n_other ? (float)k_full(it.other, a.n_other, a.alpha_other) : 0.f;
      const bool mult1 = !(J.a1 == 1.f && J.b1 == 0.f);
      // ---- stage A, input 1
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int g = 0; g < G; ++g) {
          const int c = c0 + g;
          const int kx = colkx[par][c];
          const bool slotcol = kx >= 0 && kx != it.kx0 + c;   // merged Nyquist column: global memory
          const float kc = J.ks1 == 2 ? koth : colk[c];
          const C *src = stg + n1s[h] * SPC + c + shift;
          const long long gb = (long long)it.box * a.bstride + (long long)it.other * a.otherstride + kx;
#pragma unroll
          for (int n2 = 0; n2 < N2; ++n2) {
            const int n = 64 * n2 + n1s[h];
            C v = mkc<C>(0.f, 0.f);
            if (kx >= 0 && ((rin >> (h * N2 + n2)) & 1u)) {
              v = slotcol ? J.in1[gb + (long long)n * a.rowstride] : src[64 * n2 * SPC];
              if (mult1) {
                const float bk = J.b1 * (J.ks1 == 1 ? krow[n] : kc);
                v = mkc<C>(v.x * J.a1 - v.y * bk, v.y * J.a1 + v.x * bk);
              }
            }
            z[h][g][n2] = v;
          }
        }
      if (two) {
        // ---- second input of a two-input job, staged after the first
        __syncthreads();
        if (warp == 0) {
          issue_load(i, 1);
          if (lane == 0) ++loads_issued;
        }
        if (t == 0) wait_load();
        __syncthreads();
        if (abort_s) {
          aborted = true;
          break;
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int g = 0; g < G; ++g) {
            const int c = c0 + g;
            const int kx = colkx[par][c];
            const bool slotcol = kx >= 0 && kx != it.kx0 + c;
            const float kc = J.ks2 == 2 ? koth : colk[c];
            const C *src = stg + n1s[h] * SPC + c + shift;
            const long long gb = (long long)it.box * a.bstride + (long long)it.other * a.otherstride + kx;
#pragma unroll
            for (int n2 = 0; n2 < N2; ++n2) {
              const int n = 64 * n2 + n1s[h];
              if (kx >= 0 && ((rin >> (h * N2 + n2)) & 1u)) {
                const C w2 = slotcol ? J.in2[gb + (long long)n * a.rowstride] : src[64 * n2 * SPC];
                const float bk = J.b2 * (J.ks2 == 1 ? krow[n] : kc);
                z[h][g][n2] = mkc<C>(z[h][g][n2].x + (w2.x * J.a2 - w2.y * bk),
                                     z[h][g][n2].y + (w2.y * J.a2 + w2.x * bk));
              }
            }
          }
      }
      __syncthreads();   // B0: the staging tile is consumed
      if (warp == 0 && i + 1 < my_n) {
        issue_load(i + 1, 0);
        if (lane == 0) ++loads_issued;
      }
      // ---- N2-point DFT, twiddle, column maxima
      float cmax[G];
#pragma unroll
      for (int g = 0; g < G; ++g) cmax[g] = 0.f;
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int g = 0; g < G; ++g) {
          dft<N2, C, INV>(z[h][g]);
          float m = fmaxf(fabsf(z[h][g][0].x), fabsf(z[h][g][0].y));
#pragma unroll
          for (int k2 = 1; k2 < N2; ++k2) {
            const C tw = tws[(k2 - 1) * 64 + n1s[h]];
            z[h][g][k2] = INV ? cmulc(z[h][g][k2], tw) : cmul(z[h][g][k2], tw);
            m = fmaxf(m, fmaxf(fabsf(z[h][g][k2].x), fabsf(z[h][g][k2].y)));
          }
          cmax[g] = fmaxf(cmax[g], m);
        }
#pragma unroll
      for (int g = 0; g < G; ++g) {
        // the warp's four n1 of this column group are lanes cg + 8 jq
        float m = fmaxf(cmax[g], __shfl_xor_sync(0xffffffffu, cmax[g], 8));
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 16));
        if (jq == 0) atomicMax(&pm[par][c0 + g], __float_as_uint(m));
      }
      if (t == 0 && i > 0) {   // MMA(i - 1) done: the accumulator and B are free
        if (tc::mbar_wait_bounded(&mmab, (uint32_t)(i - 1) & 1u, kTmaWaitLimit)) ++mma_seen;
        else abort_s = 3;
      }
      tc::fence_before_sync();
      __syncthreads();   // B: column maxima complete, MMA(i - 1) complete
      tc::fence_after_sync();
      if (abort_s) {
        aborted = true;
        break;
      }
    } else {
      // after the last tile: wait for its MMAs before draining
      if (t == 0 && i > 0) {
        if (tc::mbar_wait_bounded(&mmab, (uint32_t)(i - 1) & 1u, kTmaWaitLimit)) ++mma_seen;
        else abort_s = 3;
      }
      tc::fence_before_sync();
      __syncthreads();
      tc::fence_after_sync();
      if (abort_s) {
        aborted = true;
        break;
      }
    }
    // ---- drain tile i - 1 (accumulator: its MMAs are complete)
    if (i >= 1) {
      const TmaItem it = prev;
      C *obase = a.job[it.job].out + ((long long)it.box * a.bso + (long long)it.other * a.oso);
#pragma unroll
      for (int sb = 0; sb < 2; ++sb) {
        const int col0 = 64 * (warp >> 2) + 32 * sb;   // accumulator columns of this block
        const uint32_t ta = taddr + ((uint32_t)(32 * q4) << 16) + (uint32_t)col0;
        float v[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]),
              "=f"(v[8]), "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15]),
              "=f"(v[16]), "=f"(v[17]), "=f"(v[18]), "=f"(v[19]), "=f"(v[20]), "=f"(v[21]), "=f"(v[22]),
              "=f"(v[23]), "=f"(v[24]), "=f"(v[25]), "=f"(v[26]), "=f"(v[27]), "=f"(v[28]), "=f"(v[29]),
              "=f"(v[30]), "=f"(v[31])
            : "r"(ta)
            : "memory");
        tc::tmem_ld_wait();
        // unscale factors of the block's 16 pencils j = col0 / 2 + jj, column j % TCW
        float us[16];
        const float *ut = usc[par ^ 1];
        if constexpr (TCW >= 16) {
          const int cb = (col0 / 2) % TCW;
#pragma unroll
          for (int k = 0; k < 16; k += 4) {
            const float4 q = *reinterpret_cast<const float4 *>(ut + cb + k);
            us[k] = q.x, us[k + 1] = q.y, us[k + 2] = q.z, us[k + 3] = q.w;
          }
        } else {
#pragma unroll
          for (int k = 0; k < 8; k += 4) {
            const float4 q = *reinterpret_cast<const float4 *>(ut + k);
            us[k] = us[k + 8] = q.x, us[k + 1] = us[k + 9] = q.y, us[k + 2] = us[k + 10] = q.z,
                        us[k + 3] = us[k + 11] = q.w;
          }
        }
        float w[16];
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
          const float tp = __shfl_xor_sync(0xffffffffu, v[2 * jj + 1], 1);
          w[jj] = (odd ? tp + v[2 * jj] : v[2 * jj] - tp) * us[jj];
        }
        // even lane: pencils 0..7 of the block (re own, im from the odd lane); odd lane: 8..15
        float r[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) r[k] = __shfl_xor_sync(0xffffffffu, odd ? w[k] : w[8 + k], 1);
#pragma unroll
        for (int k = 0; k < 8; k += 2) {
          if (!((rout >> (4 * sb + k / 2)) & 1u)) continue;
          const int j = col0 / 2 + (odd ? 8 : 0) + k;
          const int c = j % TCW;   // even: the pair (c, c + 1) shares the output row
          const C y0 = odd ? mkc<C>(r[k], w[8 + k]) : mkc<C>(w[k], r[k]);
          const C y1 = odd ? mkc<C>(r[k + 1], w[9 + k]) : mkc<C>(w[k + 1], r[k + 1]);
          const int kxa = colkx[par ^ 1][c], kxb = colkx[par ^ 1][c + 1];
          C *orow = obase + roff[4 * sb + k / 2];
          if (kxa >= 0 && kxb >= 0 && kxa == it.kx0 + c && kxb == it.kx0 + c + 1) {
            *reinterpret_cast<float4 *>(orow + kxa) = make_float4(y0.x, y0.y, y1.x, y1.y);
          } else {
            if (kxa >= 0) orow[kxa] = y0;
            if (kxb >= 0) orow[kxb] = y1;
          }
        }
      }
    }
    if (i < my_n) {
      // ---- scale, split into f16 hi + lo, store the B operand (its last
      //      reader, MMA(i - 1), is complete)
      if (t < TCW) usc[par][t] = __int_as_float((127 + tc_exp(pm[par][t])) << 23);   // 2^e, for the drain
      float sc[G];
#pragma unroll
      for (int g = 0; g < G; ++g) sc[g] = __int_as_float((127 - tc_exp(pm[par][c0 + g])) << 23);   // 2^-e
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          __align__(16) __half2 hv[G], lv[G];
#pragma unroll
          for (int g = 0; g < G; ++g) {
            const float2 x = make_float2(z[h][g][k2].x * sc[g], z[h][g][k2].y * sc[g]);
            hv[g] = __float22half2_rn(x);
            const float2 hb = __half22float2(hv[g]);
            lv[g] = __float22half2_rn(make_float2(x.x - hb.x, x.y - hb.y));
          }
          const int off = tma::b_offset(n1s[h], 2 * (k2 * TCW + c0));
          if constexpr (G == 4) {
            *reinterpret_cast<uint4 *>(sBh + off) = *reinterpret_cast<const uint4 *>(hv);
            *reinterpret_cast<uint4 *>(sBl + off) = *reinterpret_cast<const uint4 *>(lv);
          } else if constexpr (G == 2) {
            *reinterpret_cast<uint2 *>(sBh + off) = *reinterpret_cast<const uint2 *>(hv);
            *reinterpret_cast<uint2 *>(sBl + off) = *reinterpret_cast<const uint2 *>(lv);
          } else {
            *reinterpret_cast<__half2 *>(sBh + off) = hv[0];
            *reinterpret_cast<__half2 *>(sBl + off) = lv[0];
          }
        }
      tc::fence_proxy_async();
      tc::fence_before_sync();
      __syncthreads();   // C: operands written; the drain's TMEM reads are complete
      if (t == 0) {
        tc::fence_after_sync();
        // 3 x 4 MMAs (K = 16 each) into the accumulator: Al Bh, Ah Bl, then Ah Bh
        constexpr uint32_t lboA = (128 / 8) * 128, sboA = 128, lboB = 8192, sboB = 1024;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const unsigned char *A = p == 0 ? sAl : sAh;
          const unsigned char *B = p == 1 ? sBl : sBh;
#pragma unroll
          for (int ks = 0; ks < 4; ++ks)
            tc::mma_f16(taddr, tc::smem_desc(A + 2 * ks * lboA, lboA, sboA),
                        tma::desc_sw128(B + 2 * ks * sboB, lboB, sboB), idesc, (p | ks) ? 1u : 0u);
        }
        tc::mma_commit(&mmab);
        ++mma_issued;
      }
      prev = tma_item<TCW>(a, blockIdx.x + (unsigned)i * nb);
    }
  }
  if (aborted && t == 0) {
    // wait (bounded) for the copies and MMAs still in flight before TMEM is freed
    for (int k = loads_seen; k < loads_issued; ++k) tc::mbar_wait_bounded(&full, (uint32_t)k & 1u, kTmaWaitLimit);
    for (int k = mma_seen; k < mma_issued; ++k) tc::mbar_wait_bounded(&mmab, (uint32_t)k & 1u, kTmaWaitLimit);
    atomicExch(status, abort_s);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, PL::TMEM_COLS);
}

}  // namespace dnsbox
