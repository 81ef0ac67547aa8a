// Batched 1D FFTs of length N on columns held in shared memory.
//
// Algorithm: Stockham auto-sort, mixed radix (Govindaraju et al., "High
// Performance Discrete Fourier Transforms on Graphics Processors", SC 2008):
// for a stage of radix R after sub-transforms of length Ns, butterfly b reads
// x[b + r N/R], multiplies by exp(-+2 pi i r (b mod Ns)/(Ns R)), runs an R-point
// DFT and writes y[(b/Ns) Ns R + (b mod Ns) + r Ns].  Output is in natural
// order; transforms are unnormalised (forward exp(-i..), inverse exp(+i..)).
//
// Tile layout: element (row n, column c) at s[n * LD + c]; columns are
// independent sequences.  A thread owns one column and P = N/E positions of
// it; every stage each thread holds exactly E complex values in registers
// (E/R butterflies of radix R), so register use is flat across stages.
#pragma once

#include "common.cuh"

namespace dnsbox {

// Radix schedule per transform length: E elements per thread, radices R[s].
template <int N> struct FftPlan;
#define DNSBOX_PLAN(NN, EE, ...)                                               \
  template <> struct FftPlan<NN> {                                             \
    static constexpr int N = NN;                                               \
    static constexpr int E = EE;                                               \
    static constexpr int R[] = {__VA_ARGS__};                                  \
    static constexpr int NST = sizeof(R) / sizeof(int);                        \
    __host__ __device__ static constexpr int ns(int s) { int p = 1; for (int i = 0; i < s; ++i) p *= R[i]; return p; } \
  };
DNSBOX_PLAN(8, 8, 8)
DNSBOX_PLAN(12, 12, 4, 3)
DNSBOX_PLAN(16, 16, 16)
DNSBOX_PLAN(24, 24, 8, 3)
DNSBOX_PLAN(32, 8, 8, 4)
DNSBOX_PLAN(48, 12, 4, 4, 3)
DNSBOX_PLAN(64, 8, 8, 8)
DNSBOX_PLAN(96, 12, 4, 4, 2, 3)
DNSBOX_PLAN(128, 16, 16, 8)
DNSBOX_PLAN(192, 24, 8, 8, 3)
DNSBOX_PLAN(256, 16, 16, 16)
DNSBOX_PLAN(512, 8, 8, 8, 8)
DNSBOX_PLAN(1024, 16, 16, 16, 4)
#undef DNSBOX_PLAN

// Plans with 32 threads per sequence (E = N / 32), for kernels in which one
// warp owns whole sequences and synchronises with __syncwarp only.
template <int N> struct WarpPlan;
#define DNSBOX_WPLAN(NN, EE, ...)                                              \
  template <> struct WarpPlan<NN> {                                            \
    static constexpr int N = NN;                                               \
    static constexpr int E = EE;                                               \
    static constexpr int R[] = {__VA_ARGS__};                                  \
    static constexpr int NST = sizeof(R) / sizeof(int);                        \
    __host__ __device__ static constexpr int ns(int s) { int p = 1; for (int i = 0; i < s; ++i) p *= R[i]; return p; } \
  };
DNSBOX_WPLAN(256, 8, 8, 8, 4)
DNSBOX_WPLAN(512, 16, 16, 8, 4)
DNSBOX_WPLAN(1024, 32, 16, 16, 4)
#undef DNSBOX_WPLAN

// Shared-memory addressing of element (row, col) of a tile.  Row-major tiles
// (column fastest) suit kernels whose threads run along columns; the skewed
// column-major layout suits one warp per sequence: with the skew row / R0 the
// first stage's stride-R0 writes and all consecutive-row accesses of a plan
// fall in distinct 16-byte bank groups.
struct AddrRM {
  __device__ static __forceinline__ int at(int row, int col, int ld) { return row * ld + col; }
};
template <int R0> struct AddrSkew {
  __device__ static __forceinline__ int at(int row, int col, int ld) { return col * ld + row + row / R0; }
};

template <bool WARP> __device__ __forceinline__ void fft_sync() {
  if constexpr (WARP) __syncwarp();
  else __syncthreads();
}

// ----------------------------------------------------------------- butterflies
template <typename C, bool INV> __device__ __forceinline__ void dft2(C &a, C &b) {
  C t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <typename C, bool INV> __device__ __forceinline__ void dft4(C &a0, C &a1, C &a2, C &a3) {
  C t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_i<INV>(csub(a1, a3));
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, t3);
  a3 = csub(t1, t3);
}

template <typename C, bool INV> __device__ __forceinline__ void dft3(C &a0, C &a1, C &a2) {
  using R = decltype(C{}.x);
  const R h = R(0.86602540378443864676372317075294);  // sqrt(3)/2
  C t = cadd(a1, a2), d = csub(a1, a2);
  C m = mkc<C>(a0.x - R(0.5) * t.x, a0.y - R(0.5) * t.y);
  a0 = cadd(a0, t);
  C q = mul_i<INV>(cscale(d, h));  // forward: -i h d
  a1 = cadd(m, q);
  a2 = csub(m, q);
}

// multiply by exp(-+ 2 pi i k / 8)
template <typename C, bool INV, int K> __device__ __forceinline__ C w8(C a) {
  using R = decltype(C{}.x);
  const R r = R(0.70710678118654752440084436210485);
  if constexpr (K == 0) return a;
  else if constexpr (K == 2) return mul_i<INV>(a);
  else if constexpr (K == 1) {  // (1 -+ i)/sqrt2
    return INV ? mkc<C>((a.x - a.y) * r, (a.x + a.y) * r) : mkc<C>((a.x + a.y) * r, (a.y - a.x) * r);
  } else {  // K == 3: (-1 -+ i)/sqrt2
    return INV ? mkc<C>((-a.x - a.y) * r, (a.x - a.y) * r) : mkc<C>((a.y - a.x) * r, (-a.x - a.y) * r);
  }
}

template <typename C, bool INV> __device__ __forceinline__ void dft8(C *v) {
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<C, INV>(e0, e1, e2, e3);
  dft4<C, INV>(o0, o1, o2, o3);
  o1 = w8<C, INV, 1>(o1);
  o2 = w8<C, INV, 2>(o2);
  o3 = w8<C, INV, 3>(o3);
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

// multiply by exp(-+ 2 pi i m / 16), m in [0, 9]
template <typename C, bool INV> __device__ __forceinline__ C w16(C a, int m) {
  using R = decltype(C{}.x);
  const R c1 = R(0.92387953251128675612818318939679);  // cos(pi/8)
  const R s1 = R(0.38268343236508977172845998403040);  // sin(pi/8)
  const R r = R(0.70710678118654752440084436210485);
  R c, s;  // exp(-i theta) = c - i s for forward
  switch (m) {
    case 0: return a;
    case 1: c = c1; s = s1; break;
    case 2: c = r; s = r; break;
    case 3: c = s1; s = c1; break;
    case 4: return mul_i<INV>(a);
    case 6: c = -r; s = r; break;
    case 9: c = -c1; s = -s1; break;
    default: c = 0; s = 0; break;
  }
  if (INV) s = -s;
  // (a.x + i a.y)(c - i s)
  return mkc<C>(a.x * c + a.y * s, a.y * c - a.x * s);
}

// 16-point DFT as 4 x 4: X[k1 + 4 k2] = sum_n2 W4^{n2 k2} W16^{n2 k1} sum_n1 a[4 n1 + n2] W4^{n1 k1}
template <typename C, bool INV> __device__ __forceinline__ void dft16(C *v) {
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) dft4<C, INV>(v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]);
  // now v[n2 + 4 k1] holds inner result for (n2, k1)
#pragma unroll
  for (int n2 = 1; n2 < 4; ++n2)
#pragma unroll
    for (int k1 = 1; k1 < 4; ++k1) v[n2 + 4 * k1] = w16<C, INV>(v[n2 + 4 * k1], n2 * k1);
  C o[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    C b0 = v[0 + 4 * k1], b1 = v[1 + 4 * k1], b2 = v[2 + 4 * k1], b3 = v[3 + 4 * k1];
    dft4<C, INV>(b0, b1, b2, b3);
    o[k1] = b0; o[k1 + 4] = b1; o[k1 + 8] = b2; o[k1 + 12] = b3;
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = o[i];
}

template <int R, typename C, bool INV> __device__ __forceinline__ void dft(C *v) {
  if constexpr (R == 2) dft2<C, INV>(v[0], v[1]);
  else if constexpr (R == 3) dft3<C, INV>(v[0], v[1], v[2]);
  else if constexpr (R == 4) dft4<C, INV>(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 8) dft8<C, INV>(v);
  else if constexpr (R == 16) dft16<C, INV>(v);
  else static_assert(R == 2, "unsupported radix");
}

// ----------------------------------------------------------- twiddle sources
// W_N^(r j TS) of stage S of plan PL (r in [1, R), j in [0, NS)).  TwGlobal
// reads the N-point table exp(-2 pi i k / N) through the read-only cache;
// TwShared reads per-stage [r - 1][j] tables in shared memory, so that the
// lanes of a warp with consecutive j read consecutive words (one shared
// wavefront instead of a scatter of L1 sectors), filled by tw_fill.
template <class PL, int S> __host__ __device__ constexpr int tw_off() {
  int o = 0;
  for (int t = 1; t < S; ++t) o += (PL::R[t] - 1) * PL::ns(t);
  return o;
}
template <class PL> __host__ __device__ constexpr int tw_size() { return tw_off<PL, PL::NST>(); }

template <typename C> struct TwGlobal {
  const C *__restrict__ tw;
  template <class PL, int S> __device__ __forceinline__ C get(int r, int j) const {
    constexpr int TS = PL::N / (PL::ns(S) * PL::R[S]);
    return __ldg(&tw[r * j * TS]);
  }
};
template <typename C> struct TwShared {
  const C *t;
  template <class PL, int S> __device__ __forceinline__ C get(int r, int j) const {
    return t[tw_off<PL, S>() + (r - 1) * PL::ns(S) + j];
  }
};
// Fills the shared tables of plan PL from the global N-point table (all
// threads of the block take part; the caller synchronises afterwards).
template <typename C, class PL, int S = 1>
__device__ __forceinline__ void tw_fill(C *t, const C *__restrict__ tw, int tid, int nthreads) {
  if constexpr (S < PL::NST) {
    constexpr int NS = PL::ns(S), R = PL::R[S], TS = PL::N / (NS * R);
    for (int i = tid; i < (R - 1) * NS; i += nthreads) {
      const int r = 1 + i / NS, j = i % NS;
      t[tw_off<PL, S>() + i] = tw[r * j * TS];
    }
    tw_fill<C, PL, S + 1>(t, tw, tid, nthreads);
  }
}

// ----------------------------------------------------------------- stages
// One Stockham stage on column `col` of the tile; p in [0, N/E).  All threads
// of the block call it (barriers inside); `active` masks idle threads.
template <typename C, class PL, int S, bool INV, bool WARP, class AD = AddrRM, class TW = TwGlobal<C>>
__device__ __forceinline__ void fft_stage_p(C *s, int LD, int col, int p, bool active, const TW &tw) {
  constexpr int N = PL::N;
  constexpr int R = PL::R[S];
  constexpr int NS = PL::ns(S);
  constexpr int E = PL::E;
  constexpr int NB = N / R;
  constexpr int P = N / E;
  constexpr int M = E / R;
  C v[M][R];
  if (active) {
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int b = p + m * P;
#pragma unroll
      for (int r = 0; r < R; ++r) v[m][r] = s[AD::at(b + r * NB, col, LD)];
    }
  }
  fft_sync<WARP>();
  if (active) {
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int b = p + m * P;
      const int j = b % NS;
      if constexpr (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const C w = tw.template get<PL, S>(r, j);
          v[m][r] = INV ? cmulc(v[m][r], w) : cmul(v[m][r], w);
        }
      }
      dft<R, C, INV>(v[m]);
      const int o = (b / NS) * NS * R + j;
#pragma unroll
      for (int r = 0; r < R; ++r) s[AD::at(o + r * NS, col, LD)] = v[m][r];
    }
  }
  fft_sync<WARP>();
}

template <typename C, int N, int S, bool INV>
__device__ __forceinline__ void fft_stage(C *s, int LD, int col, int p, bool active, const C *__restrict__ tw) {
  fft_stage_p<C, FftPlan<N>, S, INV, false>(s, LD, col, p, active, TwGlobal<C>{tw});
}

template <typename C, int N, bool INV, int S = 0>
__device__ __forceinline__ void fft_columns(C *s, int LD, int col, int p, bool active,
                                            const C *__restrict__ tw) {
  if constexpr (S < FftPlan<N>::NST) {
    fft_stage<C, N, S, INV>(s, LD, col, p, active, tw);
    fft_columns<C, N, INV, S + 1>(s, LD, col, p, active, tw);
  }
}

// ------------------------------------------------- register-resident ends
// A thread's E values are v[m * R + r] for butterfly b = p + m P (P = N/E)
// and leg r.  The first stage reads rows b + r N/R0 and the last stage writes
// rows b + r N/RL: for consecutive p these are consecutive rows, so a caller
// can load the first stage's inputs straight from global memory and store the
// last stage's outputs straight back, with only the middle exchanges in
// shared memory.
template <class PL> struct FftEndsP {
  static constexpr int N = PL::N;
  static constexpr int E = PL::E;
  static constexpr int P = N / E;
  static constexpr int R0 = PL::R[0];
  static constexpr int RL = PL::R[PL::NST - 1];
  static constexpr int NB0 = N / R0;
  static constexpr int NBL = N / RL;
  __device__ static __forceinline__ int in_row(int p, int i) { return p + (i / R0) * P + (i % R0) * NB0; }
  __device__ static __forceinline__ int out_row(int p, int i) { return p + (i / RL) * P + (i % RL) * NBL; }
};
template <int N> using FftEnds = FftEndsP<FftPlan<N>>;

// Stage 0 on registers (no twiddles since Ns = 1), result stored to shared
// memory in Stockham order, then a barrier.  For a single-stage plan the
// result stays in v (in out_row order) and nothing touches shared memory.
template <typename C, class PL, bool INV, bool WARP, class AD = AddrRM>
__device__ __forceinline__ void fft_first_regs_p(C *v, C *s, int LD, int col, int p, bool active) {
  constexpr int N = PL::N;
  constexpr int R = PL::R[0];
  constexpr int M = PL::E / R;
  constexpr int P = N / PL::E;
  if (active) {
#pragma unroll
    for (int m = 0; m < M; ++m) dft<R, C, INV>(v + m * R);
  }
  if constexpr (PL::NST > 1) {
    if (active) {
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int b = p + m * P;
#pragma unroll
        for (int r = 0; r < R; ++r) s[AD::at(b * R + r, col, LD)] = v[m * R + r];
      }
    }
    fft_sync<WARP>();
  }
}

// Last stage from shared memory into registers (v in out_row order).  The
// caller owns the barrier that must follow before shared memory is reused.
template <typename C, class PL, bool INV, class AD = AddrRM, class TW = TwGlobal<C>>
__device__ __forceinline__ void fft_last_regs_p(C *v, const C *s, int LD, int col, int p, bool active,
                                                const TW &tw) {
  constexpr int N = PL::N;
  constexpr int S = PL::NST - 1;
  constexpr int R = PL::R[S];
  constexpr int NS = PL::ns(S);
  constexpr int NB = N / R;
  constexpr int P = N / PL::E;
  constexpr int M = PL::E / R;
  if (!active) return;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int b = p + m * P;
#pragma unroll
    for (int r = 0; r < R; ++r) v[m * R + r] = s[AD::at(b + r * NB, col, LD)];
    const int j = b % NS;
#pragma unroll
    for (int r = 1; r < R; ++r) {
      const C w = tw.template get<PL, S>(r, j);
      v[m * R + r] = INV ? cmulc(v[m * R + r], w) : cmul(v[m * R + r], w);
    }
    dft<R, C, INV>(v + m * R);
  }
}

// Stages 1 .. NST-2 in shared memory.
template <typename C, class PL, bool INV, bool WARP, class AD = AddrRM, int S = 1, class TW = TwGlobal<C>>
__device__ __forceinline__ void fft_middle_p(C *s, int LD, int col, int p, bool active, const TW &tw) {
  if constexpr (S + 1 < PL::NST) {
    fft_stage_p<C, PL, S, INV, WARP, AD, TW>(s, LD, col, p, active, tw);
    fft_middle_p<C, PL, INV, WARP, AD, S + 1, TW>(s, LD, col, p, active, tw);
  }
}

// Whole transform with v holding the first stage's inputs on entry and the
// last stage's outputs on exit.  Shared memory (N x LD tile) is scratch;
// ends with a barrier (block or warp) so the tile may be reused.
template <typename C, class PL, bool INV, bool WARP, class AD = AddrRM, class TW>
__device__ __forceinline__ void fft_regs_t(C *v, C *s, int LD, int col, int p, bool active, const TW &tw) {
  fft_first_regs_p<C, PL, INV, WARP, AD>(v, s, LD, col, p, active);
  if constexpr (PL::NST > 1) {
    fft_middle_p<C, PL, INV, WARP, AD, 1, TW>(s, LD, col, p, active, tw);
    fft_last_regs_p<C, PL, INV, AD, TW>(v, s, LD, col, p, active, tw);
    fft_sync<WARP>();
  }
}
template <typename C, class PL, bool INV, bool WARP, class AD = AddrRM>
__device__ __forceinline__ void fft_regs_p(C *v, C *s, int LD, int col, int p, bool active,
                                           const C *__restrict__ tw) {
  fft_regs_t<C, PL, INV, WARP, AD>(v, s, LD, col, p, active, TwGlobal<C>{tw});
}

template <typename C, int N, bool INV>
__device__ __forceinline__ void fft_regs(C *v, C *s, int LD, int col, int p, bool active,
                                         const C *__restrict__ tw) {
  fft_regs_p<C, FftPlan<N>, INV, false>(v, s, LD, col, p, active, tw);
}

}  // namespace dnsbox
