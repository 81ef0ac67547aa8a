// Launchers of the size-templated pass kernels.  Each (precision, N) pair is
// explicitly instantiated in its own translation unit (inst.cu built once per
// pair), so the library compiles in parallel; api.cu sees declarations only.
#pragma once

#include <type_traits>

#include "kernels.cuh"
#include "kernels_tc.cuh"
#include "kernels_tma.cuh"

namespace dnsbox {

template <typename T, int N> struct Launcher {
  static cudaError_t strided(const StridedArgs<T> &a, bool inv, int ntiles, cudaStream_t st);
  // tensor-core split-precision form of `strided` (FP32, N = 128 .. 1024);
  // adft: the four DFT-64 operands, status: set to 1 if an MMA wait gave up
  static cudaError_t strided_tc(const StridedArgs<T> &a, bool inv, int nother, const void *adft, int *status,
                                int nctas, cudaStream_t st);
  static bool has_tc();
  // TMA-staged tensor-core pass of the right-hand side (FP32, N = 128 .. 512)
  static cudaError_t strided_tma(const TmaArgs &a, bool inv, const void *adft, int *status, int nctas,
                                 cudaStream_t st);
  static bool has_tma();
  // variant: 0 the default kernel for N, 1 the block kernel, 2 the warp kernel, 3 the warp kernel with
  // each line's fields in registers (N = 256, FP32), 4 the same held to the registers of four resident
  // blocks per SM; 3 and 4 run the warp kernel at other sizes
  static cudaError_t xline_nl(const XlineNLArgs<T> &a, int variant, cudaStream_t st);
  static bool has_xline_warp();
  static cudaError_t xline_c2r(const XlineArgs<T> &a, int nf, cudaStream_t st);
  static cudaError_t xline_r2c(const XlineArgs<T> &a, int nf, cudaStream_t st);
  static int strided_threads();
};

#define DNSBOX_SIZES(X) X(8) X(12) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(512) X(1024)

#ifdef DNSBOX_LAUNCH_IMPL
// Opts the kernel in to `bytes` of dynamic shared memory (the 48 KB default
// covers static + dynamic, so it is set for every size); refuses sizes over
// the 227 KB per-CTA limit.
template <typename K>
static cudaError_t set_smem(K kernel, size_t bytes) {
  if (bytes > 227 * 1024) return cudaErrorInvalidConfiguration;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename T, int N> int Launcher<T, N>::strided_threads() {
  return round32(StridedCols<T, N>::v * (N / FftPlan<N>::E));
}

template <typename T, int N>
cudaError_t Launcher<T, N>::strided(const StridedArgs<T> &a, bool inv, int ntiles, cudaStream_t st) {
  using C = typename CT<T>::type;
  const size_t smem = (size_t)N * StridedCols<T, N>::v * sizeof(C);
  const int nt = strided_threads();
  const dim3 nb((unsigned)ntiles * a.njobs * (TileCols<T>::v / StridedCols<T, N>::v),
                (unsigned)(a.nbatch > 0 ? a.nbatch : 1));
  cudaError_t e;
  if (inv) {
    if ((e = set_smem(k_strided<T, N, true>, smem)) != cudaSuccess) return e;
    k_strided<T, N, true><<<nb, nt, smem, st>>>(a);
  } else {
    if ((e = set_smem(k_strided<T, N, false>, smem)) != cudaSuccess) return e;
    k_strided<T, N, false><<<nb, nt, smem, st>>>(a);
  }
  return cudaGetLastError();
}

template <typename T, int N> bool Launcher<T, N>::has_tc() {
  return std::is_same<T, float>::value && TcPlan<N>::on;
}

template <typename T, int N>
cudaError_t Launcher<T, N>::strided_tc(const StridedArgs<T> &a, bool inv, int nother, const void *adft,
                                       int *status, int nctas, cudaStream_t st) {
  if constexpr (std::is_same<T, float>::value && TcPlan<N>::on) {
    using PL = TcPlan<N>;
    TcArgs g;
    g.ntx = strided_ntx(a, PL::TCW);   // column tiles of the (possibly pruned) grid
    g.nother = nother;
    const long long total = (long long)a.njobs * g.ntx * nother * (a.nbatch > 0 ? a.nbatch : 1);
    if (total == 0) return cudaSuccess;
    if (total + 2LL * nctas >= (1LL << 31)) return cudaErrorInvalidValue;
    if ((long long)N * a.rowstride >= (1LL << 31) || (long long)N * out_rowstride(a) >= (1LL << 31))
      return cudaErrorInvalidValue;   // 32-bit row offsets
    g.total = (int)total;
    g.per_box.init((unsigned)(a.njobs * g.ntx * nother));
    g.njobs.init((unsigned)a.njobs);
    g.ntxd.init((unsigned)g.ntx);
    const unsigned nb = (unsigned)(g.total < nctas ? g.total : nctas);
    const __half *A = reinterpret_cast<const __half *>(adft) + (inv ? 2 * 128 * 64 : 0);
    cudaError_t e;
    // two 96 KB CTAs per SM: ask for the largest shared-memory carveout
    if ((e = cudaFuncSetAttribute(inv ? k_strided_tc<N, true> : k_strided_tc<N, false>,
                                  cudaFuncAttributePreferredSharedMemoryCarveout, 100)) != cudaSuccess)
      return e;
    if (inv) {
      if ((e = set_smem(k_strided_tc<N, true>, PL::SMEM)) != cudaSuccess) return e;
      k_strided_tc<N, true><<<nb, PL::THREADS, PL::SMEM, st>>>(a, g, A, status);
    } else {
      if ((e = set_smem(k_strided_tc<N, false>, PL::SMEM)) != cudaSuccess) return e;
      k_strided_tc<N, false><<<nb, PL::THREADS, PL::SMEM, st>>>(a, g, A, status);
    }
    return cudaGetLastError();
  } else {
    (void)a, (void)inv, (void)nother, (void)adft, (void)status, (void)nctas, (void)st;
    return cudaErrorInvalidValue;
  }
}

template <typename T, int N> bool Launcher<T, N>::has_tma() {
  return std::is_same<T, float>::value && TmaPlan<N>::on;
}

template <typename T, int N>
cudaError_t Launcher<T, N>::strided_tma(const TmaArgs &a, bool inv, const void *adft, int *status, int nctas,
                                        cudaStream_t st) {
  if constexpr (std::is_same<T, float>::value && TmaPlan<N>::on) {
    using PL = TmaPlan<N>;
    if (a.total == 0) return cudaSuccess;
    const unsigned nb = (unsigned)(a.total < nctas ? a.total : nctas);
    const __half *A = reinterpret_cast<const __half *>(adft) + (inv ? 2 * 128 * 64 : 0);
    cudaError_t e;
    // two CTAs of ~105 KB per SM: ask for the largest shared-memory carveout
    if ((e = cudaFuncSetAttribute(inv ? k_strided_tma<N, true> : k_strided_tma<N, false>,
                                  cudaFuncAttributePreferredSharedMemoryCarveout, 100)) != cudaSuccess)
      return e;
    if (inv) {
      if ((e = set_smem(k_strided_tma<N, true>, PL::SMEM)) != cudaSuccess) return e;
      k_strided_tma<N, true><<<nb, PL::THREADS, PL::SMEM, st>>>(a, A, status);
    } else {
      if ((e = set_smem(k_strided_tma<N, false>, PL::SMEM)) != cudaSuccess) return e;
      k_strided_tma<N, false><<<nb, PL::THREADS, PL::SMEM, st>>>(a, A, status);
    }
    return cudaGetLastError();
  } else {
    (void)a, (void)inv, (void)adft, (void)status, (void)nctas, (void)st;
    return cudaErrorInvalidValue;
  }
}

template <typename T, int N> bool Launcher<T, N>::has_xline_warp() { return XlineWarp<T, N>::on; }

template <typename T, int N>
cudaError_t Launcher<T, N>::xline_nl(const XlineNLArgs<T> &a, int variant, cudaStream_t st) {
  using C = typename CT<T>::type;
  if constexpr (XlineWarp<T, N>::on) {
    if (variant != 1) {
    // warp-granular kernel: one warp per line pair
    constexpr int WPB = XlineWarp<T, N>::wpb;
    constexpr int LDC = N + N / XlineWarp<T, N>::Plan::R[0];
    const size_t smem = ((size_t)WPB * 6 * LDC + XlineWarp<T, N>::twn) * sizeof(C);
    cudaError_t e;
    const long long pairs = (a.nlines + 1) / 2;
    const unsigned nb = (unsigned)((pairs + WPB - 1) / WPB);
    if constexpr (N == 256 && sizeof(T) == 4) {
      if (variant == 3 || variant == 4) {
        // fields of a line in registers: two exchange columns per warp (4: held to
        // 128 registers for four blocks per SM)
        const size_t smem_r = ((size_t)WPB * 2 * LDC + XlineWarp<T, N>::twn) * sizeof(C);
        auto kern = variant == 3 ? k_xline_nl_r<T> : k_xline_nl_r<T, 4>;
        if ((e = set_smem(kern, smem_r)) != cudaSuccess) return e;
        kern<<<nb, 32 * WPB, smem_r, st>>>(a);
        return cudaGetLastError();
      }
    }
    if ((e = set_smem(k_xline_nl_w<T, N>, smem)) != cudaSuccess) return e;
    k_xline_nl_w<T, N><<<nb, 32 * WPB, smem, st>>>(a);
    return cudaGetLastError();
    }
  }
  constexpr int B = XlineB<T, N>::v;
  const size_t smem = (size_t)N * (3 * B + 1) * sizeof(C);
  const int nt = round32(3 * B * (N / FftPlan<N>::E));
  cudaError_t e;
  if ((e = set_smem(k_xline_nl<T, N>, smem)) != cudaSuccess) return e;
  const unsigned nb = (unsigned)((a.nlines + B - 1) / B);
  k_xline_nl<T, N><<<nb, nt, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int N>
cudaError_t Launcher<T, N>::xline_c2r(const XlineArgs<T> &a, int nf, cudaStream_t st) {
  using C = typename CT<T>::type;
  constexpr int B = XlinePlainB<T, N>::v;
  const size_t smem = (size_t)N * (B / 2 + 1) * sizeof(C);
  const int nt = round32((B / 2) * (N / FftPlan<N>::E));
  cudaError_t e;
  if ((e = set_smem(k_xline_c2r<T, N>, smem)) != cudaSuccess) return e;
  dim3 grid((unsigned)((a.nlines + B - 1) / B), (unsigned)nf);
  k_xline_c2r<T, N><<<grid, nt, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int N>
cudaError_t Launcher<T, N>::xline_r2c(const XlineArgs<T> &a, int nf, cudaStream_t st) {
  using C = typename CT<T>::type;
  constexpr int B = XlinePlainB<T, N>::v;
  const size_t smem = (size_t)N * (B / 2 + 1) * sizeof(C);
  const int nt = round32((B / 2) * (N / FftPlan<N>::E));
  cudaError_t e;
  if ((e = set_smem(k_xline_r2c<T, N>, smem)) != cudaSuccess) return e;
  dim3 grid((unsigned)((a.nlines + B - 1) / B), (unsigned)nf);
  k_xline_r2c<T, N><<<grid, nt, smem, st>>>(a);
  return cudaGetLastError();
}

#endif

}  // namespace dnsbox
