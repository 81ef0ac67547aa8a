// Pass kernels of the dnsbox B200 pseudospectral step.
//
// Every spectral or mixed-space array is [nz][ny][nxh] complex with the kx
// (half-axis) index fastest; physical arrays are [nz][ny][nx] real.  A 3D
// transform is three passes, one per axis:
//   z and y : k_strided  -- tiles of TC consecutive kx columns x N rows along
//             the axis; each CTA runs one "job" (one output field) whose input
//             is in1*(a1 + i b1 k) + in2*(a2 + i b2 k), which fuses the spectral
//             curl into the inverse transforms;
//   x       : k_xline_*  -- whole lines along x, two real lines per complex FFT.
// The nonlinear term fuses the last inverse x pass, the u x omega product, the
// max|u_i| (CFL) reduction and the first forward x pass (k_xline_nl); after
// the last forward z pass (k_strided, in place) one streaming kernel applies
// dealiasing, pressure projection, band forcing, the integrating-factor
// stepper and the energy/dissipation row sums (k_finish_rows).
#pragma once

#include <type_traits>

#include "common.cuh"
#include "fft.cuh"

namespace dnsbox {

// Blocks are launched with a multiple of 32 threads (full warps for the
// shuffle reductions); threads beyond the FFT's own count only take part in
// the strided element loops and barriers.
__host__ __device__ constexpr int round32(int x) { return (x + 31) / 32 * 32; }
// Resident CTAs to ask the register allocator for: `want` for blocks of up
// to 256 threads, one for larger blocks (which hold enough warps alone).
__host__ __device__ constexpr int min_ctas(int threads, int want) { return threads <= 256 ? want : 1; }

// Host/device step bookkeeping kept in device memory (one per context).
struct StepState {
  double dt;        // step size of the current step
  double t;         // time at the start of the current step
  double t_prev;    // time at the start of the previous step (AB2 history)
  double eband;     // rhs_Eband of the current RHS input
  double umax[3];   // max |u_i| of the current RHS input (atomic max)
  double courant;   // io_Courant of the step's initial state with dt
  double eband1;    // eband of the step's first RHS (for the diagnostics)
  double step;      // step counter
  double pad[6];
};

// Pruning of the 2/3-rule zeros.  On an axis of length n the dealiasing mask
// (rhs.f90:74-88) keeps index i when |k_i| < (n/2)(2/3) alpha, i.e. i < a, the
// Nyquist index n/2 (whose wavenumber is 0) and, on full axes, i > n - a.  A
// state that vanishes outside the kept set keeps doing so under the stepper,
// so the transforms may skip loading those zeros, skip outputs the mask
// discards, and skip whole tiles; results are bit-identical.  a = 0: no pruning.
struct AxisKeep {
  int a, n, full;
  __host__ __device__ __forceinline__ bool keep(int i) const {
    return a == 0 || i < a || i == (n >> 1) || (full && i > n - a);
  }
  // kept indices of a full axis in order: [0, a), n/2, (n - a, n)
  __host__ __device__ __forceinline__ int count() const { return a == 0 ? n : 2 * a; }
  __host__ __device__ __forceinline__ int map(int o) const {
    return (a == 0 || o < a) ? o : (o == a ? (n >> 1) : n - 2 * a + o);
  }
};

// Tile width (kx columns) of the strided passes: 128 B per row segment.
template <typename T> struct TileCols;
template <> struct TileCols<double> { static constexpr int v = 8; };
template <> struct TileCols<float> { static constexpr int v = 16; };

template <typename T> struct StridedJob {
  using C = typename CT<T>::type;
  const C *in1;
  const C *in2;
  C *out;
  double a1, b1, a2, b2;   // multiplier a + i b k
  int ks1, ks2;            // k: 0 kx of the column, 1 the row index's, 2 the tile's other-axis index's
};

template <typename T> struct StridedArgs {
  using C = typename CT<T>::type;
  StridedJob<T> job[6];
  const C *tw;             // exp(-2 pi i j / N), j < N
  int njobs;
  int ncols;               // nxh
  int nx;
  int pad0;
  long long rowstride;     // elements between consecutive rows of the axis
  long long otherstride;   // elements between consecutive tiles of the other axis
  double alpha_row, alpha_x;
  int n_other;             // length of the other axis (for ks = 2)
  int nbatch;              // boxes (blockIdx.y), each job pointer advanced by bstride per box
  double alpha_other;
  long long bstride;
  // pruning (all zero when off, so zero-initialised arguments run the full
  // grid): kept kx columns, kept other-axis indices (the tile grid covers only
  // these), kept input rows (others read as 0) and kept output rows (others
  // not stored).  Column tiles: all ceil(ncols / width) when ntx_lo = 0, else
  // [0, ntx_lo) followed by tile nyq_tile when nyq_tile > 0; nyq_tile < 0
  // places the Nyquist column in the free slot kx = kcol.a of the last low
  // tile (see strided_col).
  AxisKeep kcol, koth, krin, krout;
  int ntx_lo, nyq_tile;
  // strides of the output when its row pitch differs from the input's (the
  // padded workspace fields of a right-hand side); 0: the input's
  long long rowstride_o, otherstride_o, bstride_o;
};

// Output strides of a strided launch (the input's where unset).
template <typename T> __host__ __device__ __forceinline__ long long out_rowstride(const StridedArgs<T> &a) {
  return a.rowstride_o ? a.rowstride_o : a.rowstride;
}
template <typename T> __host__ __device__ __forceinline__ long long out_otherstride(const StridedArgs<T> &a) {
  return a.otherstride_o ? a.otherstride_o : a.otherstride;
}
template <typename T> __host__ __device__ __forceinline__ long long out_bstride(const StridedArgs<T> &a) {
  return a.bstride_o ? a.bstride_o : a.bstride;
}

// Column tiles of the grid of a strided launch with tile width tcw.
template <typename T>
__host__ __device__ __forceinline__ int strided_ntx(const StridedArgs<T> &a, int tcw) {
  return a.ntx_lo ? a.ntx_lo + (a.nyq_tile > 0 ? 1 : 0) : (a.ncols + tcw - 1) / tcw;
}

// Half-axis index held by tile column kx0 + c: the identity, except in the
// merged layout (nyq_tile < 0), where the first column past the cut holds the
// Nyquist column kcol.n / 2.
template <typename T>
__host__ __device__ __forceinline__ int strided_col(const StridedArgs<T> &a, int kx) {
  return (a.nyq_tile < 0 && kx == a.kcol.a) ? (a.kcol.n >> 1) : kx;
}

// Columns per CTA of the SIMT strided kernel: the host's tile width, or at
// N >= 512 (plans of 64 threads per column) half a tile, so that a CTA has
// 512 (FP32) or 256 (FP64) threads and several CTAs share an SM, each with
// its own barriers; in FP32 at every size (at 256: 128-thread CTAs, eight per
// SM, 5% off the inverse y pass at 256^3; at 96 the pruned 34-column grid
// wastes 6 columns instead of 14, 3% off the 96^3 strided passes; the FP64
// kernel below 512 keeps its tile).
template <typename T, int N> struct StridedCols {
  static constexpr int v = (N >= 512 || sizeof(T) == 4) ? TileCols<T>::v / 2 : TileCols<T>::v;
};

// Resident CTAs of a strided launch to ask the register allocator for: FP32
// blocks of up to 256 threads whose plans hold at most 16 values a thread
// are held to 64 registers a thread (the load-latency-bound passes gain more
// from the extra warps than they lose to the tighter allocation), 512-thread
// FP32 blocks to two per SM and the 256-thread FP64 blocks of N = 512 to
// three (80 registers, a few spills: 24% off the inverse y pass at 512^3);
// 0 leaves the choice to the compiler.
template <typename T, int N> struct StridedMinCtas {
  static constexpr int NT = round32(StridedCols<T, N>::v * (N / FftPlan<N>::E));
  static constexpr int v = (sizeof(T) == 4 && NT <= 256 && FftPlan<N>::E <= 16) ? 1024 / NT
                         : (sizeof(T) == 4 && NT == 512) ? 2 : (sizeof(T) == 8 && N == 512) ? 3 : 0;
};

// Column origin and other-axis index of tile t of the (possibly pruned) grid.
template <typename T>
__device__ __forceinline__ void strided_tile(const StridedArgs<T> &a, int tile, int tcw, int &kx0, int &other) {
  const int ntk = strided_ntx(a, tcw);
  const int o = tile / ntk, kt = tile - o * ntk;
  kx0 = (a.ntx_lo == 0 || kt < a.ntx_lo ? kt : a.nyq_tile) * tcw;
  other = a.koth.map(o);
}

template <typename T, typename C>
__device__ __forceinline__ C apply_mult(C v, double a, double b, double k) {
  // v * (a + i b k)
  const T bk = T(b * k), aa = T(a);
  return mkc<C>(v.x * aa - v.y * bk, v.y * aa + v.x * bk);
}

template <typename T, int N, bool INV>
__global__ void __launch_bounds__(round32(StridedCols<T, N>::v *(N / FftPlan<N>::E)), StridedMinCtas<T, N>::v)
    k_strided(const __grid_constant__ StridedArgs<T> a) {
  using C = typename CT<T>::type;
  using EN = FftEnds<N>;
  constexpr int TC = StridedCols<T, N>::v;    // columns of this CTA
  constexpr int SPLIT = TileCols<T>::v / TC;  // CTAs per tile of the host's grid
  constexpr int E = EN::E;
  constexpr int NF = TC * (N / E);   // FFT threads: column fastest
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s = reinterpret_cast<C *>(smem_raw);
  // block (tile, job, part): the parts of a tile are adjacent blocks, so they
  // read the two halves of the same 128-byte row segments at about one time
  const int part = blockIdx.x % SPLIT, tj = blockIdx.x / SPLIT;
  const int job = tj % a.njobs;
  const int tile = tj / a.njobs;
  int kx0, other;
  strided_tile(a, tile, TileCols<T>::v, kx0, other);
  kx0 += part * TC;
  // the job's fields, read from the parameter bank once (an indexed
  // parameter read each time they are used measured as a busy ADU pipe)
  const C *const in1p = a.job[job].in1, *const in2p = a.job[job].in2;
  C *const outp = a.job[job].out;
  const double ja1 = a.job[job].a1, jb1 = a.job[job].b1, ja2 = a.job[job].a2, jb2 = a.job[job].b2;
  const int ks1 = a.job[job].ks1, ks2 = a.job[job].ks2;
  const bool act = threadIdx.x < NF;
  const int col = threadIdx.x % TC, p = threadIdx.x / TC;
  const int kx = strided_col(a, kx0 + col);
  const bool valid = act && kx < a.ncols && a.kcol.keep(kx);
  const long long base = (long long)other * a.otherstride + kx + (long long)blockIdx.y * a.bstride;
  // FP32: the job's row multipliers T(b k_row(n)) (ks == 1), once per block
  // instead of once per element (the same values as apply_mult forms; FP64
  // evaluates them per element, which keeps its kernel at 128 registers)
  constexpr bool TAB = sizeof(T) == 4;
  __shared__ T bks[2][TAB ? N : 1];
  const bool mult1 = !(ja1 == 1.0 && jb1 == 0.0);
  if (TAB && ((mult1 && ks1 == 1) || (in2p && ks2 == 1))) {
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
      const double k = k_full(n, N, a.alpha_row);
      bks[0][n] = T(jb1 * k);
      bks[1][n] = T(jb2 * k);
    }
    __syncthreads();
  }
  C v[E];
  if (valid) {
    // all E loads of the first stage are independent and issued together
    const C *in1 = in1p + base;
#pragma unroll
    for (int i = 0; i < E; ++i)
      v[i] = a.krin.keep(EN::in_row(p, i)) ? in1[(long long)EN::in_row(p, i) * a.rowstride] : mkc<C>(0, 0);
    // wavenumber of the column (0) or of the tile's other-axis index (2)
    const double kcol = k_half(kx, a.nx, a.alpha_x);
    const double koth = a.n_other ? k_full(other, a.n_other, a.alpha_other) : 0.0;
    if constexpr (TAB) {
      if (mult1) {
        const T aa = T(ja1), bkc = T(jb1 * (ks1 == 2 ? koth : kcol));
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const T bk = ks1 == 1 ? bks[0][EN::in_row(p, i)] : bkc;
          v[i] = mkc<C>(v[i].x * aa - v[i].y * bk, v[i].y * aa + v[i].x * bk);
        }
      }
      if (in2p) {
        const C *in2 = in2p + base;
        const T aa = T(ja2), bkc = T(jb2 * (ks2 == 2 ? koth : kcol));
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const C w = a.krin.keep(EN::in_row(p, i)) ? in2[(long long)EN::in_row(p, i) * a.rowstride] : mkc<C>(0, 0);
          const T bk = ks2 == 1 ? bks[1][EN::in_row(p, i)] : bkc;
          v[i] = cadd(v[i], mkc<C>(w.x * aa - w.y * bk, w.y * aa + w.x * bk));
        }
      }
    } else {
      if (mult1) {
        const double kc = ks1 == 2 ? koth : kcol;
#pragma unroll
        for (int i = 0; i < E; ++i)
          v[i] = apply_mult<T>(v[i], ja1, jb1, ks1 == 1 ? k_full(EN::in_row(p, i), N, a.alpha_row) : kc);
      }
      if (in2p) {
        const C *in2 = in2p + base;
        const double kc = ks2 == 2 ? koth : kcol;
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const C w = a.krin.keep(EN::in_row(p, i)) ? in2[(long long)EN::in_row(p, i) * a.rowstride] : mkc<C>(0, 0);
          v[i] = cadd(v[i], apply_mult<T>(w, ja2, jb2, ks2 == 1 ? k_full(EN::in_row(p, i), N, a.alpha_row) : kc));
        }
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = mkc<C>(0, 0);
  }
  fft_regs<C, N, INV>(v, s, TC, col, p, act, a.tw);
  if (valid) {
    const long long rso = out_rowstride(a);
    C *out = outp + ((long long)other * out_otherstride(a) + kx + (long long)blockIdx.y * out_bstride(a));
#pragma unroll
    for (int i = 0; i < E; ++i)
      if (a.krout.keep(EN::out_row(p, i))) out[(long long)EN::out_row(p, i) * rso] = v[i];
  }
}

// ------------------------------------------------------------------ x lines
template <typename T> struct XlineNLArgs {
  using C = typename CT<T>::type;
  const C *U, *V, *W, *OX, *OY, *OZ;  // (kx, y, z) space, rows of nxh; omega scaled by 1/N^3
  C *NX, *NY, *NZ;                     // forward x transforms of (omega x u) * s
  const C *tw;
  StepState *st;                       // per-box step state: umax[3] gets max |u_i| (true scale)
  int nlines, nxh;
  int lines_per_box;                   // ny * nz
  int kxa;                             // pruning: only kx < kxa and kx = N/2 are read and written (0: all)
  int pin, pout;                       // row pitch (complex elements) of the inputs / outputs; 0: nxh
  int *status;                         // set to 1 when a bounded wait of a staged kernel gives up (or null)
  double alpha_x;
  double s;                            // scalemodes
};

// kept half-axis index under the x-line pruning rule
__device__ __forceinline__ bool xkeep(int kxa, int k, int n) { return kxa == 0 || k < kxa || k == (n >> 1); }

// Lines per CTA of the fused x pass (even; 3B columns in shared memory).  In
// FP32 below 256, 8 where 16 lines would make 384-thread blocks (N = 64, 96,
// 128): four 192-thread CTAs per SM instead of two of 384, each with its own
// barriers (x pass 10-13% faster at 64^3 and 96^3).
template <typename T, int N> struct XlineB {
  static constexpr int v = (N >= 512) ? 2
                         : (sizeof(T) == 8 ? (N >= 256 ? 4 : 8)
                                           : (N >= 256 || (FftPlan<N>::E <= 16 && 3 * 16 * (N / FftPlan<N>::E) > 256)
                                                  ? 8 : 16));
};

// Full-length sequence value at row n of Z = X1 + i X2, where X1, X2 are the
// half spectra (nxh values) of two real lines: rows above N/2 are the
// Hermitian mirror; the imaginary parts of the kx = 0 and Nyquist bins are
// dropped, as a C2R does.
template <typename C, int N>
__device__ __forceinline__ C pack_pair(int n, C X1, C X2) {
  if (n == 0 || n == N / 2) return mkc<C>(X1.x, X2.x);
  if (n < N / 2) return mkc<C>(X1.x - X2.y, X1.y + X2.x);
  return mkc<C>(X1.x + X2.y, X2.x - X1.y);   // conj(X1) + i conj(X2) at N - n
}

// Resident CTAs of the block x-line kernel to ask the register allocator
// for: 3 for blocks of up to 256 threads; 2 for the 384-thread FP32 blocks of
// N = 1024 (80 registers instead of 123, two CTAs per SM instead of one).
template <typename T, int N> struct XlineMinCtas {
  static constexpr int NT = round32(3 * XlineB<T, N>::v * (N / FftPlan<N>::E));
  static constexpr int v = (sizeof(T) == 4 && N >= 1024) ? 2 : min_ctas(NT, 3);
};

template <typename T, int N>
__global__ void __launch_bounds__(round32(3 * XlineB<T, N>::v *(N / FftPlan<N>::E)), XlineMinCtas<T, N>::v)
    k_xline_nl(const __grid_constant__ XlineNLArgs<T> a) {
  using C = typename CT<T>::type;
  using EN = FftEnds<N>;
  constexpr int B = XlineB<T, N>::v;
  constexpr int H = N / 2 + 1;
  constexpr int NCOL = 3 * B;
  constexpr int LD = NCOL + 1;         // odd stride: rows fall in distinct bank groups
  constexpr int E = EN::E;
  constexpr int P = N / E;
  constexpr int NF = NCOL * P;         // FFT threads, position index fastest
  constexpr int NQ = NCOL / 2;         // forward sequences
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s = reinterpret_cast<C *>(smem_raw);
  __shared__ double red[3 * 32];
  const int NT = blockDim.x;
  const int line0 = blockIdx.x * B;
  const T sc = T(a.s);
  // Inverse transforms.  Column 6j+q of line pair (a = 2j, b = 2j+1) holds
  // (u_a,v_a) (u_b,v_b) (w_a,w_b) (ox_a,oy_a) (ox_b,oy_b) (oz_a,oz_b): each
  // pair is two quantities of the same kind and scale.
  {
    const bool act = threadIdx.x < NF;
    const int p = threadIdx.x % P, col = threadIdx.x / P;
    const int j = col / 6, q = col % 6;
    const int la = line0 + 2 * j, lb = la + 1;
    const C *f1, *f2;
    int l1, l2;
    switch (q) {
      case 0: f1 = a.U; l1 = la; f2 = a.V; l2 = la; break;
      case 1: f1 = a.U; l1 = lb; f2 = a.V; l2 = lb; break;
      case 2: f1 = a.W; l1 = la; f2 = a.W; l2 = lb; break;
      case 3: f1 = a.OX; l1 = la; f2 = a.OY; l2 = la; break;
      case 4: f1 = a.OX; l1 = lb; f2 = a.OY; l2 = lb; break;
      default: f1 = a.OZ; l1 = la; f2 = a.OZ; l2 = lb; break;
    }
    const bool v1 = act && l1 < a.nlines, v2 = act && l2 < a.nlines;
    const long long pin = a.pin ? a.pin : a.nxh;
    const C *r1 = f1 + (long long)l1 * pin, *r2 = f2 + (long long)l2 * pin;
    C v[E];
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const int n = EN::in_row(p, i);
      const int kk = n <= N / 2 ? n : N - n;
      const bool kp = xkeep(a.kxa, kk, N);
      const C X1 = (v1 && kp) ? r1[kk] : mkc<C>(0, 0);
      const C X2 = (v2 && kp) ? r2[kk] : mkc<C>(0, 0);
      v[i] = pack_pair<C, N>(n, X1, X2);
    }
    fft_regs<C, N, true>(v, s, LD, col, p, act, a.tw);
    if (act) {
#pragma unroll
      for (int i = 0; i < E; ++i) s[EN::out_row(p, i) * LD + col] = v[i];
    }
  }
  __syncthreads();
  // (omega x u) * s at every point; written back as (px_a,py_a) (pz_a,pz_b)
  // (px_b,py_b) in columns 6j, 6j+1, 6j+2; the CFL maxima are taken in T
  // (exact) and widened for the block reduction
  T m0 = 0, m1 = 0, m2 = 0;
  for (int it = threadIdx.x; it < N * (B / 2); it += NT) {
    const int n = it % N, j = it / N;
    C *r = s + n * LD + 6 * j;
    const C c0 = r[0], c1 = r[1], c2 = r[2], c3 = r[3], c4 = r[4], c5 = r[5];
    const T uu[2] = {c0.x, c1.x}, vv[2] = {c0.y, c1.y}, ww[2] = {c2.x, c2.y};
    const T ox[2] = {c3.x, c4.x}, oy[2] = {c3.y, c4.y}, oz[2] = {c5.x, c5.y};
    T px[2], py[2], pz[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      px[h] = (oy[h] * ww[h] - oz[h] * vv[h]) * sc;
      py[h] = (oz[h] * uu[h] - ox[h] * ww[h]) * sc;
      pz[h] = (ox[h] * vv[h] - oy[h] * uu[h]) * sc;
      m0 = fmax(m0, fabs(uu[h]));
      m1 = fmax(m1, fabs(vv[h]));
      m2 = fmax(m2, fabs(ww[h]));
    }
    r[0] = mkc<C>(px[0], py[0]);
    r[1] = mkc<C>(pz[0], pz[1]);
    r[2] = mkc<C>(px[1], py[1]);
  }
  __syncthreads();
  // forward transforms of the NQ product sequences
  {
    const bool act = threadIdx.x < NQ * P;
    const int p = threadIdx.x % P, q = threadIdx.x / P;
    const int col = 6 * (q / 3) + q % 3;
    C v[E];
    if (act) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = s[EN::in_row(p, i) * LD + col];
    }
    __syncthreads();
    fft_regs<C, N, false>(v, s, LD, col, p, act, a.tw);
    if (act) {
#pragma unroll
      for (int i = 0; i < E; ++i) s[EN::out_row(p, i) * LD + col] = v[i];
    }
  }
  __syncthreads();
  // unpack two real transforms per sequence and store
  const long long pout = a.pout ? a.pout : a.nxh;
  for (int it = threadIdx.x; it < NQ * H; it += NT) {
    const int k = it % H, q = it / H;
    const int j = q / 3, c = q % 3;
    const int col = 6 * j + c;
    const C zk = s[k * LD + col], zn = s[((N - k) % N) * LD + col];
    const C X1 = mkc<C>(T(0.5) * (zk.x + zn.x), T(0.5) * (zk.y - zn.y));
    const C X2 = mkc<C>(T(0.5) * (zk.y + zn.y), T(-0.5) * (zk.x - zn.x));
    const int la = line0 + 2 * j, lb = la + 1;
    if (!xkeep(a.kxa, k, N)) continue;
    if (c == 0) {
      if (la < a.nlines) {
        a.NX[(long long)la * pout + k] = X1;
        a.NY[(long long)la * pout + k] = X2;
      }
    } else if (c == 1) {
      if (la < a.nlines) a.NZ[(long long)la * pout + k] = X1;
      if (lb < a.nlines) a.NZ[(long long)lb * pout + k] = X2;
    } else {
      if (lb < a.nlines) {
        a.NX[(long long)lb * pout + k] = X1;
        a.NY[(long long)lb * pout + k] = X2;
      }
    }
  }
  // CFL reduction
  m0 = warp_max(m0);
  m1 = warp_max(m1);
  m2 = warp_max(m2);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[wid] = (double)m0;
    red[32 + wid] = (double)m1;
    red[64 + wid] = (double)m2;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = NT >> 5;
    double x0 = lane < nw ? red[lane] : 0, x1 = lane < nw ? red[32 + lane] : 0,
           x2 = lane < nw ? red[64 + lane] : 0;
    x0 = warp_max(x0);
    x1 = warp_max(x1);
    x2 = warp_max(x2);
    if (lane == 0 && a.st) {
      // B divides ny*nz, so every line of the CTA belongs to one box
      double *um = a.st[line0 / a.lines_per_box].umax;
      atomic_max_nonneg(um + 0, x0 * a.s);
      atomic_max_nonneg(um + 1, x1 * a.s);
      atomic_max_nonneg(um + 2, x2 * a.s);
    }
  }
}

// Warp-granular variant of the fused x pass for N >= 256: each warp owns one
// line pair from its loads to its stores and synchronises only with
// __syncwarp, so the SM overlaps one warp's memory phases with another's
// transforms (the block-wide barriers of k_xline_nl serialise them).  Columns
// of a warp's tile are the six sequences of k_xline_nl, stored column-major
// with the row / R0 skew (conflict-free for both plans below).  At N = 256 a
// sequence runs the two-stage radix-16 plan on 16 threads, so a warp
// transforms two sequences at once with one shared-memory exchange each; at
// N = 512 a sequence runs the three-stage plan on all 32 threads.
// In FP32 the twiddles come from per-stage tables in shared memory (one
// wavefront per lane-varying read instead of a scatter of L1 sectors, which
// left the kernel bound by L1 throughput); FP64 keeps the global table, whose
// shared copy would cost a resident block.
template <typename T, int N> struct XlineWarp {
  static constexpr bool on = N == 256 || N == 512;
  static constexpr int wpb = sizeof(T) == 8 ? (N >= 512 ? 1 : 2) : (N >= 1024 ? 1 : (N >= 512 ? 2 : 4));
  using Plan = typename std::conditional<N == 256, FftPlan<256>, WarpPlan<N>>::type;
  static constexpr bool full3 = 32 / (N / Plan::E) == 2 && sizeof(T) == 4;   // see xline_w_tail
  static constexpr bool smtw = on && sizeof(T) == 4;
  static constexpr int twn = smtw ? tw_size<Plan>() + (full3 ? tw_size<WarpPlan<N>>() : 0) : 0;
  // twiddle tables of the block after its warps' tiles; all threads fill them
  __device__ static __forceinline__ typename CT<T>::type *tables(unsigned char *smem, const typename CT<T>::type *tw,
                                                                  int cols = 6) {
    using C = typename CT<T>::type;
    C *t = reinterpret_cast<C *>(smem) + (size_t)wpb * cols * (N + N / Plan::R[0]);
    if constexpr (smtw) {
      tw_fill<C, Plan>(t, tw, threadIdx.x, blockDim.x);
      if constexpr (full3) tw_fill<C, WarpPlan<N>>(t + tw_size<Plan>(), tw, threadIdx.x, blockDim.x);
      __syncthreads();
    }
    return t;
  }
};

// The x pass's transform of `v` on column `col` with the kernel's twiddle source.
template <typename T, class PL, bool INV, class AD, int N>
__device__ __forceinline__ void xw_fft(typename CT<T>::type *v, typename CT<T>::type *s, int LD, int col, int p,
                                       bool active, const typename CT<T>::type *tw, const typename CT<T>::type *twt) {
  using C = typename CT<T>::type;
  if constexpr (XlineWarp<T, N>::smtw) fft_regs_t<C, PL, INV, true, AD>(v, s, LD, col, p, active, TwShared<C>{twt});
  else fft_regs_p<C, PL, INV, true, AD>(v, s, LD, col, p, active, tw);
}

// Second half of the warp-granular fused x pass for one line pair (la, lb):
// the inverse transforms are in the warp's tile s (column-major, skewed);
// (omega x u) * s, the three forward transforms, the unpacking into the
// output half lines and the CFL maxima of the pair.
template <typename T, int N>
__device__ __forceinline__ void xline_w_tail(typename CT<T>::type *s, const XlineNLArgs<T> &a, long long la,
                                             long long lb, int lane, long long pout,
                                             const typename CT<T>::type *twt) {
  using C = typename CT<T>::type;
  using PL = typename XlineWarp<T, N>::Plan;
  using EN = FftEndsP<PL>;
  using AD = AddrSkew<PL::R[0]>;
  constexpr int E = PL::E;
  constexpr int P = N / E;
  constexpr int SPW = 32 / P;
  constexpr int H = N / 2 + 1;
  constexpr int LDC = N + N / PL::R[0];
  const int p = lane % P, h = lane / P;
  const T sc = T(a.s);
  __syncwarp();
  // (omega x u) * s, written back as (px_a,py_a) (pz_a,pz_b) (px_b,py_b) in
  // columns 0..2; the CFL maxima are taken in T (exact) and widened at the end
  T m0 = 0, m1 = 0, m2 = 0;
#pragma unroll 4
  for (int n = lane; n < N; n += 32) {
    const C c0 = s[AD::at(n, 0, LDC)], c1 = s[AD::at(n, 1, LDC)], c2 = s[AD::at(n, 2, LDC)];
    const C c3 = s[AD::at(n, 3, LDC)], c4 = s[AD::at(n, 4, LDC)], c5 = s[AD::at(n, 5, LDC)];
    const T uu[2] = {c0.x, c1.x}, vv[2] = {c0.y, c1.y}, ww[2] = {c2.x, c2.y};
    const T ox[2] = {c3.x, c4.x}, oy[2] = {c3.y, c4.y}, oz[2] = {c5.x, c5.y};
    T px[2], py[2], pz[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      px[h] = (oy[h] * ww[h] - oz[h] * vv[h]) * sc;
      py[h] = (oz[h] * uu[h] - ox[h] * ww[h]) * sc;
      pz[h] = (ox[h] * vv[h] - oy[h] * uu[h]) * sc;
      m0 = fmax(m0, fabs(uu[h]));
      m1 = fmax(m1, fabs(vv[h]));
      m2 = fmax(m2, fabs(ww[h]));
    }
    s[AD::at(n, 0, LDC)] = mkc<C>(px[0], py[0]);
    s[AD::at(n, 1, LDC)] = mkc<C>(pz[0], pz[1]);
    s[AD::at(n, 2, LDC)] = mkc<C>(px[1], py[1]);
  }
  __syncwarp();
  // forward transforms of the three product sequences, SPW at a time.  In
  // FP32 with two per warp, sequence 2 runs on all 32 lanes with the 32-thread
  // plan (same column, skew and twiddle table) instead of on one half-warp
  // (in FP64 that form measured slower)
  constexpr bool FULL3 = XlineWarp<T, N>::full3;
  constexpr int RF = FULL3 ? 1 : (3 + SPW - 1) / SPW;
#pragma unroll 1
  for (int r = 0; r < RF; ++r) {
    const int q = SPW * r + h;
    const bool act = q < 3;
    const int qc = act ? q : 0;
    C v[E];
    if (act) {
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = s[AD::at(EN::in_row(p, i), qc, LDC)];
    }
    __syncwarp();
    xw_fft<T, PL, false, AD, N>(v, s, LDC, qc, p, act, a.tw, twt);
    if (act) {
#pragma unroll
      for (int i = 0; i < E; ++i) s[AD::at(EN::out_row(p, i), qc, LDC)] = v[i];
    }
  }
  if constexpr (FULL3) {
    using WP = WarpPlan<N>;
    using EW = FftEndsP<WP>;
    static_assert(N + (N - 1) / PL::R[0] < LDC, "the 32-thread plan stays inside its column");
    C w[WP::E];
#pragma unroll
    for (int i = 0; i < WP::E; ++i) w[i] = s[AD::at(EW::in_row(lane, i), 2, LDC)];
    __syncwarp();
    xw_fft<T, WP, false, AD, N>(w, s, LDC, 2, lane, true, a.tw, twt + tw_size<PL>());
#pragma unroll
    for (int i = 0; i < WP::E; ++i) s[AD::at(EW::out_row(lane, i), 2, LDC)] = w[i];
  }
  __syncwarp();
  // unpack two real transforms per sequence and store
  for (int k = lane; k < H; k += 32) {
    if (!xkeep(a.kxa, k, N)) continue;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const C zk = s[AD::at(k, q, LDC)], zn = s[AD::at((N - k) % N, q, LDC)];
      const C X1 = mkc<C>(T(0.5) * (zk.x + zn.x), T(0.5) * (zk.y - zn.y));
      const C X2 = mkc<C>(T(0.5) * (zk.y + zn.y), T(-0.5) * (zk.x - zn.x));
      if (q == 0) {
        a.NX[la * pout + k] = X1;
        a.NY[la * pout + k] = X2;
      } else if (q == 1) {
        a.NZ[la * pout + k] = X1;
        a.NZ[lb * pout + k] = X2;
      } else {
        a.NX[lb * pout + k] = X1;
        a.NY[lb * pout + k] = X2;
      }
    }
  }
  // CFL maxima of this line pair (both lines lie in one box: ny*nz is even)
  m0 = warp_max(m0);
  m1 = warp_max(m1);
  m2 = warp_max(m2);
  if (lane == 0 && a.st) {
    double *um = a.st[la / a.lines_per_box].umax;
    atomic_max_nonneg(um + 0, (double)m0 * a.s);
    atomic_max_nonneg(um + 1, (double)m1 * a.s);
    atomic_max_nonneg(um + 2, (double)m2 * a.s);
  }
}

template <typename T, int N>
__global__ void __launch_bounds__(32 * XlineWarp<T, N>::wpb)
    k_xline_nl_w(const __grid_constant__ XlineNLArgs<T> a) {
  using C = typename CT<T>::type;
  using PL = typename XlineWarp<T, N>::Plan;
  using EN = FftEndsP<PL>;
  using AD = AddrSkew<PL::R[0]>;
  constexpr int E = PL::E;
  constexpr int P = N / E;                // threads per sequence
  constexpr int SPW = 32 / P;             // sequences a warp transforms at once
  constexpr int LDC = N + N / PL::R[0];   // column length with the skew
  constexpr int WPB = XlineWarp<T, N>::wpb;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C *s = reinterpret_cast<C *>(smem_raw) + (size_t)warp * 6 * LDC;
  const C *twt = XlineWarp<T, N>::tables(smem_raw, a.tw);   // (a block barrier in FP32)
  const long long la = 2 * ((long long)blockIdx.x * WPB + warp), lb = la + 1;
  if (la >= a.nlines) return;
  const C *f1s[6] = {a.U, a.U, a.W, a.OX, a.OX, a.OZ};
  const C *f2s[6] = {a.V, a.V, a.W, a.OY, a.OY, a.OZ};
  const long long l1s[6] = {la, lb, la, la, lb, la};
  const long long l2s[6] = {la, lb, lb, la, lb, lb};
  const int p = lane % P, h = lane / P;   // position in the sequence, sequence slot
  const long long pin = a.pin ? a.pin : a.nxh, pout = a.pout ? a.pout : a.nxh;
  // inverse transforms: round r transforms sequences SPW r + h; the loads of
  // the next round are issued before this round's transform.  A lane loads
  // only its rows n = p + P i <= N/2 (i < E/2, and i = E/2 at p = 0); row
  // N - n of the Hermitian mirror is row n' = (P - p) + P (E - 1 - i) of lane
  // P - p (lane p = 0: its own row P (E - i)), taken by a shuffle, so every
  // half-line element is read from global memory once.
  static_assert(PL::R[0] == E, "first-stage rows n = p + P i");
  C x1[E], x2[E];
  auto load = [&](const C *g1, const C *g2) {
#pragma unroll
    for (int i = 0; i <= E / 2; ++i) {
      const int n = p + P * i;   // <= N / 2 for i < E / 2 and for p = 0
      const bool kp = (i < E / 2 || p == 0) && xkeep(a.kxa, n, N);
      x1[i] = kp ? g1[n] : mkc<C>(0, 0);
      x2[i] = kp ? g2[n] : mkc<C>(0, 0);
    }
  };
  const int mirror = (lane & ~(P - 1)) | ((P - p) & (P - 1));   // lane of the mirror rows
  auto mirror_fill = [&]() {
#pragma unroll
    for (int i = E / 2; i < E; ++i) {
      const int j = E - 1 - i;
      C m1 = mkc<C>(__shfl_sync(0xffffffffu, x1[j].x, mirror), __shfl_sync(0xffffffffu, x1[j].y, mirror));
      C m2 = mkc<C>(__shfl_sync(0xffffffffu, x2[j].x, mirror), __shfl_sync(0xffffffffu, x2[j].y, mirror));
      if (p == 0) {   // rows 0 and N/2 are its own loads; N - P i = P (E - i)
        m1 = i == E / 2 ? x1[i] : x1[E - i];
        m2 = i == E / 2 ? x2[i] : x2[E - i];
      }
      x1[i] = m1;
      x2[i] = m2;
    }
  };
  load(f1s[h] + l1s[h] * pin, f2s[h] + l2s[h] * pin);
#pragma unroll 1
  for (int r = 0; r < 6 / SPW; ++r) {
    const int q = SPW * r + h;
    C v[E];
    mirror_fill();
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = pack_pair<C, N>(EN::in_row(p, i), x1[i], x2[i]);
    if (r + 1 < 6 / SPW) {
      const int qn = q + SPW;
      load(f1s[qn] + l1s[qn] * pin, f2s[qn] + l2s[qn] * pin);
    }
    xw_fft<T, PL, true, AD, N>(v, s, LDC, q, p, true, a.tw, twt);
#pragma unroll
    for (int i = 0; i < E; ++i) s[AD::at(EN::out_row(p, i), q, LDC)] = v[i];
  }
  xline_w_tail<T, N>(s, a, la, lb, lane, pout, twt);
}

// Plain x-line transforms of nf fields (blockIdx.y = field).
// Fused x pass at N = 256 with the fields of a line in registers (FP32).
// Half-warp h owns line la + h and packs its six real lines as three
// sequences, U + iV, W + i 2^e OZ and OX + i OY, transformed one per round on
// its 16 lanes.  With the two-stage radix-16 plan a lane's first-stage
// input rows and last-stage output rows are the same, n = p + 16 i, so after
// the three rounds every lane holds u, v, w and the vorticity at its 16
// rows: the cross product and the CFL maxima need no shared memory, and the
// products px + i py are already the forward transform's inputs.  The third
// forward sequence, pz(a) + i pz(b), is formed by one shuffle across the
// halves and transformed by both (each stores its line's half).  Shared
// memory holds only each sequence's one exchange (two columns per warp) and
// the twiddle tables.  Hermitian-mirror rows, on input and output, come from
// the partner lane by shuffle.
// MINB > 0: that many resident blocks per SM asked of the register allocator.
template <typename T, int MINB = 0>
__global__ void __launch_bounds__(32 * XlineWarp<T, 256>::wpb, MINB)
    k_xline_nl_r(const __grid_constant__ XlineNLArgs<T> a) {
  constexpr int N = 256;
  using C = typename CT<T>::type;
  using PL = typename XlineWarp<T, N>::Plan;
  using EN = FftEndsP<PL>;
  using AD = AddrSkew<PL::R[0]>;
  constexpr int E = PL::E;
  constexpr int P = N / E;
  static_assert(P == 16 && E == 16 && PL::NST == 2 && PL::R[0] == 16 && PL::R[1] == 16,
                "rows n = p + 16 i at both ends of the transform");
  constexpr int LDC = N + N / PL::R[0];
  constexpr int WPB = XlineWarp<T, N>::wpb;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = lane & 15, h = lane >> 4;
  C *s = reinterpret_cast<C *>(smem_raw) + (size_t)warp * 2 * LDC;
  const C *twt = XlineWarp<T, N>::tables(smem_raw, a.tw, 2);   // (a block barrier in FP32)
  const long long la = 2 * ((long long)blockIdx.x * WPB + warp);
  if (la >= a.nlines) return;
  const long long line = la + h;
  const long long pin = a.pin ? a.pin : a.nxh, pout = a.pout ? a.pout : a.nxh;
  const T sc = T(a.s);
  const int mirror = (lane & 16) | ((16 - p) & 15);
  // rows n = p + 16 i <= N / 2 of the two half lines of a sequence
  C x1[E / 2 + 1], x2[E / 2 + 1];
  auto load = [&](const C *g1, const C *g2) {
#pragma unroll
    for (int i = 0; i <= E / 2; ++i) {
      const int n = p + P * i;
      const bool kp = (i < E / 2 || p == 0) && xkeep(a.kxa, n, N);
      x1[i] = kp ? g1[n] : mkc<C>(0, 0);
      x2[i] = kp ? g2[n] : mkc<C>(0, 0);
    }
  };
  // value at row N - (p + 16 i) of a lane's rows from w (own rows): the partner
  // lane's row p' + 16 (15 - i), or (p = 0) its own row 16 (16 - i)
  auto shfl_c = [&](C c, int src) {
    return mkc<C>(__shfl_sync(0xffffffffu, c.x, src), __shfl_sync(0xffffffffu, c.y, src));
  };
  const C *f1s[3] = {a.U, a.W, a.OX};
  const C *f2s[3] = {a.V, a.OZ, a.OY};
  // W and OZ share a sequence, and the vorticity is larger than the velocity
  // by the factor s of the spectral curl and by the wavenumbers of the field:
  // the transform would round OZ's part relative to W's, so each line's OZ is
  // first brought to its W's magnitude by a power of two (exact both ways),
  // the exponent difference of the two half lines' largest components.
  T up = 1, down = 1;
  C o[3][E];   // inverse transforms: (u, v), (w, 2^e oz), (ox, oy) at rows p + 16 i
  load(f1s[0] + line * pin, f2s[0] + line * pin);
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    C v[E];
    if (r == 1) {
      T mw = 0, mo = 0;
#pragma unroll
      for (int i = 0; i <= E / 2; ++i) {
        mw = fmax(mw, fmax(fabs(x1[i].x), fabs(x1[i].y)));
        mo = fmax(mo, fmax(fabs(x2[i].x), fabs(x2[i].y)));
      }
#pragma unroll
      for (int o = 8; o; o >>= 1) {   // the 16 lanes of this line
        mw = fmax(mw, __shfl_xor_sync(0xffffffffu, mw, o));
        mo = fmax(mo, __shfl_xor_sync(0xffffffffu, mo, o));
      }
      int ew = 0, eo = 0;
      frexp(mw, &ew);
      frexp(mo, &eo);
      const int d = mw > 0 && mo > 0 ? max(-96, min(96, ew - eo)) : 0;
      up = ldexp(T(1), d);
      down = ldexp(T(1), -d);
#pragma unroll
      for (int i = 0; i <= E / 2; ++i) x2[i] = mkc<C>(x2[i].x * up, x2[i].y * up);
    }
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const int n = p + P * i;
      C y1, y2;
      if (i < E / 2) {
        y1 = x1[i], y2 = x2[i];
      } else {
        y1 = shfl_c(x1[E - 1 - i], mirror);
        y2 = shfl_c(x2[E - 1 - i], mirror);
        if (p == 0) {
          y1 = i == E / 2 ? x1[E / 2] : x1[E - i];
          y2 = i == E / 2 ? x2[E / 2] : x2[E - i];
        }
      }
      v[i] = pack_pair<C, N>(n, y1, y2);
    }
    if (r < 2) load(f1s[r + 1] + line * pin, f2s[r + 1] + line * pin);
    xw_fft<T, PL, true, AD, N>(v, s, LDC, h, p, true, a.tw, twt);
#pragma unroll
    for (int i = 0; i < E; ++i) o[r][i] = v[i];
  }
  // (omega x u) s at the lane's rows, and the CFL maxima
  T m0 = 0, m1 = 0, m2 = 0;
  C f[E];
  T pz[E];
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const T u = o[0][i].x, v = o[0][i].y, w = o[1][i].x, oz = o[1][i].y * down, ox = o[2][i].x, oy = o[2][i].y;
    f[i] = mkc<C>((oy * w - oz * v) * sc, (oz * u - ox * w) * sc);
    pz[i] = (ox * v - oy * u) * sc;
    m0 = fmax(m0, fabs(u));
    m1 = fmax(m1, fabs(v));
    m2 = fmax(m2, fabs(w));
  }
  // forward transforms and the unpacking of two real transforms per sequence:
  // X1[k] = (Z[k] + conj Z[N-k]) / 2, X2[k] = (Z[k] - conj Z[N-k]) / 2i at k = p + 16 i <= N/2
  auto unpack_store = [&](const C *z, C *d1, C *d2) {
#pragma unroll
    for (int i = 0; i <= E / 2; ++i) {
      const int k = p + P * i;
      C zn = shfl_c(z[(E - 1 - i) & (E - 1)], mirror);
      if (p == 0) zn = z[(E - i) & (E - 1)];
      const C zk = z[i];
      if ((i < E / 2 || p == 0) && xkeep(a.kxa, k, N)) {
        if (d1) d1[k] = mkc<C>(T(0.5) * (zk.x + zn.x), T(0.5) * (zk.y - zn.y));
        if (d2) d2[k] = mkc<C>(T(0.5) * (zk.y + zn.y), T(-0.5) * (zk.x - zn.x));
      }
    }
  };
  xw_fft<T, PL, false, AD, N>(f, s, LDC, h, p, true, a.tw, twt);
  unpack_store(f, a.NX + line * pout, a.NY + line * pout);
  // pz(a) + i pz(b) on both halves (the same sequence)
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const T other = __shfl_xor_sync(0xffffffffu, pz[i], 16);
    f[i] = h == 0 ? mkc<C>(pz[i], other) : mkc<C>(other, pz[i]);
  }
  xw_fft<T, PL, false, AD, N>(f, s, LDC, h, p, true, a.tw, twt);
  unpack_store(f, h == 0 ? a.NZ + line * pout : nullptr, h == 1 ? a.NZ + line * pout : nullptr);
  // CFL maxima of the pair (both lines lie in one box: ny*nz is even)
  m0 = warp_max(m0);
  m1 = warp_max(m1);
  m2 = warp_max(m2);
  if (lane == 0 && a.st) {
    double *um = a.st[la / a.lines_per_box].umax;
    atomic_max_nonneg(um + 0, (double)m0 * a.s);
    atomic_max_nonneg(um + 1, (double)m1 * a.s);
    atomic_max_nonneg(um + 2, (double)m2 * a.s);
  }
}

template <typename T> struct XlineArgs {
  using C = typename CT<T>::type;
  const void *in[6];
  void *out[6];
  const C *tw;
  int nlines, nxh;
  double scale;            // multiplies the output
};

template <typename T, int N> struct XlinePlainB {
  static constexpr int v = (sizeof(T) == 8 ? 16 : 32) / ((N >= 512) ? 4 : 1);
};

// C2R along x: half lines (nxh complex) -> real lines (N), two lines per FFT.
template <typename T, int N>
__global__ void __launch_bounds__(round32((XlinePlainB<T, N>::v / 2) * (N / FftPlan<N>::E)))
    k_xline_c2r(const __grid_constant__ XlineArgs<T> a) {
  using C = typename CT<T>::type;
  using EN = FftEnds<N>;
  constexpr int B = XlinePlainB<T, N>::v;
  constexpr int NC = B / 2;
  constexpr int LD = NC + 1;
  constexpr int E = EN::E;
  constexpr int P = N / E;
  constexpr int NF = NC * P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s = reinterpret_cast<C *>(smem_raw);
  const C *in = reinterpret_cast<const C *>(a.in[blockIdx.y]);
  T *out = reinterpret_cast<T *>(a.out[blockIdx.y]);
  const bool act = threadIdx.x < NF;
  const int p = threadIdx.x % P, j = threadIdx.x / P;
  const int la = blockIdx.x * B + 2 * j, lb = la + 1;
  const bool va = act && la < a.nlines, vb = act && lb < a.nlines;
  C v[E];
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int n = EN::in_row(p, i);
    const int kk = n <= N / 2 ? n : N - n;
    const C X1 = va ? in[(long long)la * a.nxh + kk] : mkc<C>(0, 0);
    const C X2 = vb ? in[(long long)lb * a.nxh + kk] : mkc<C>(0, 0);
    v[i] = pack_pair<C, N>(n, X1, X2);
  }
  fft_regs<C, N, true>(v, s, LD, j, p, act, a.tw);
  const T sc = T(a.scale);
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int n = EN::out_row(p, i);
    if (va) out[(long long)la * N + n] = v[i].x * sc;
    if (vb) out[(long long)lb * N + n] = v[i].y * sc;
  }
}

// R2C along x: real lines -> half lines, two lines per FFT.
template <typename T, int N>
__global__ void __launch_bounds__(round32((XlinePlainB<T, N>::v / 2) * (N / FftPlan<N>::E)))
    k_xline_r2c(const __grid_constant__ XlineArgs<T> a) {
  using C = typename CT<T>::type;
  using EN = FftEnds<N>;
  constexpr int B = XlinePlainB<T, N>::v;
  constexpr int NC = B / 2;
  constexpr int LD = NC + 1;
  constexpr int H = N / 2 + 1;
  constexpr int E = EN::E;
  constexpr int P = N / E;
  constexpr int NF = NC * P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s = reinterpret_cast<C *>(smem_raw);
  const T *in = reinterpret_cast<const T *>(a.in[blockIdx.y]);
  C *out = reinterpret_cast<C *>(a.out[blockIdx.y]);
  const int NT = blockDim.x;
  const bool act = threadIdx.x < NF;
  const int p = threadIdx.x % P, j = threadIdx.x / P;
  const int line0 = blockIdx.x * B;
  {
    const int la = line0 + 2 * j, lb = la + 1;
    const bool va = act && la < a.nlines, vb = act && lb < a.nlines;
    C v[E];
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const int n = EN::in_row(p, i);
      v[i] = mkc<C>(va ? in[(long long)la * N + n] : T(0), vb ? in[(long long)lb * N + n] : T(0));
    }
    fft_regs<C, N, false>(v, s, LD, j, p, act, a.tw);
    if (act) {
#pragma unroll
      for (int i = 0; i < E; ++i) s[EN::out_row(p, i) * LD + j] = v[i];
    }
  }
  __syncthreads();
  const T sc = T(a.scale);
  for (int it = threadIdx.x; it < NC * H; it += NT) {
    const int k = it % H, jj = it / H;
    const int la = line0 + 2 * jj, lb = la + 1;
    const C zk = s[k * LD + jj], zn = s[((N - k) % N) * LD + jj];
    const C X1 = mkc<C>(T(0.5) * (zk.x + zn.x) * sc, T(0.5) * (zk.y - zn.y) * sc);
    const C X2 = mkc<C>(T(0.5) * (zk.y + zn.y) * sc, T(-0.5) * (zk.x - zn.x) * sc);
    if (la < a.nlines) out[(long long)la * a.nxh + k] = X1;
    if (lb < a.nlines) out[(long long)lb * a.nxh + k] = X2;
  }
}

// ------------------------------------------------------------- z finish
enum FinishMode : int {
  FIN_RHS = 0,         // out <- N(u)
  FIN_PRED = 1,        // out <- IF (uin + dt N); nold <- N if nold
  FIN_CORR = 2,        // state <- 0.5 (IF state + uin) + 0.5 dt N
  FIN_AB2 = 3,         // state(=uin) <- IF uin + c1 IF N + c2 E2 nold; nold <- N
};

template <typename T> struct FinishArgs {
  using C = typename CT<T>::type;
  const C *n3;             // 3 fields (kx, ky, kz): the nonlinear term after the forward z pass
  const C *uin;            // 3 fields, RHS input (forcing)
  C *out;                  // FIN_RHS / FIN_PRED output (3 fields)
  C *state;                // FIN_CORR state (3 fields)
  C *nold;                 // AB2 history (3 fields)
  const C *force;          // fixed spectral forcing added to N (3 fields) or null
  const StepState *st;     // per-box step state (blockIdx.y)
  const double *nu_box;    // per-box viscosity or null (use nu)
  double *partials;        // per-CTA (E, D) of the new state, or null; gridDim.x pairs per box
  const C *tw;
  long long nh;            // elements between components (all boxes of one component)
  long long bstride;       // elements between boxes
  int nx, ny, nz, nxh;
  double ax, ay, az;
  double nu, Q, Pin, kcut;
  double cutx, cuty, cutz, sph2;
  int bandlim, spherical, mode, ab2_standard;
  double s;                // scalemodes
  AxisKeep kx, ky, kz;     // pruning: only kept (kz, ky) rows and kept kx modes are visited
  // layout of n3 when it is a padded workspace field: row pitch, elements
  // between components and between boxes; 0: the state's (nxh, nh, bstride)
  int n3_pitch;
  long long n3_nh, n3_bstride;
  // a ky slab of a box split over ranks: row ky of this launch is ky0 + ky of
  // an axis of ny_k rows (0, 0: the box's own rows)
  int ky0, ny_k;
};

// Spectral finish after the forward z transform (the second half of one
// right-hand side's pass E): per mode the 2/3 mask, the pressure projection,
// band or fixed forcing and the integrating-factor update, one warp per
// (kz, ky) row of kx modes.  n3 holds the z-transformed nonlinear term.  Rows
// run over the kept kz and ky indices (every row when not pruning) and cut kx
// modes are skipped; the row's E and D sums (fixed lane order) go to
// partials[kz ny + ky] of the box, and the finalize reads the rows a pruned
// launch does not visit as zero.  Each lane batches the global operands of
// two modes before any store.  MODE (a FinishMode) is a template parameter so
// that only the operands of the update in use occupy registers.
// Resident blocks per SM asked of the register allocator: the FP32
// corrector and AB2 finishes (115-120 registers, two blocks) are held to
// three blocks.
template <typename T, int MODE> struct FinishMinB {
  static constexpr int v = (sizeof(T) == 4 && (MODE == 2 || MODE == 3)) ? 3 : 0;
};

template <typename T, int MODE>
__global__ void __launch_bounds__(256, FinishMinB<T, MODE>::v)
    k_finish_rows(const __grid_constant__ FinishArgs<T> a, int nrows) {
  using C = typename CT<T>::type;
  constexpr int CH = 2;
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= nrows) return;   // whole warps: no block-level synchronisation below
  const int nky = a.ky.count();
  const int oz = w / nky;
  const int kz = a.kz.map(oz), ky = a.ky.map(w - oz * nky);
  const int box = blockIdx.y;
  const long long rowbase = ((long long)kz * a.ny + ky) * a.nxh + (long long)box * a.bstride;
  const long long n3nh = a.n3_nh ? a.n3_nh : a.nh;
  const long long n3row = ((long long)kz * a.ny + ky) * (a.n3_pitch ? a.n3_pitch : a.nxh) +
                          (long long)box * (a.n3_bstride ? a.n3_bstride : a.bstride);
  const StepState *st = a.st + box;
  const double nu = a.nu_box ? a.nu_box[box] : a.nu;
  const double dt = st->dt;
  const double fc = a.bandlim ? a.Pin / (2.0 * st->eband) : 0.0;
  double c1 = 0, c2 = 0, tau2 = 0;
  if (MODE == FIN_AB2) {
    const double tn = st->t, tm = st->t_prev;
    if (a.ab2_standard) {
      const double h = tn - tm;
      c1 = dt * (1.0 + dt / (2.0 * h));
      c2 = -dt * dt / (2.0 * h);
    } else {  // dnsbox.f90:150-161
      c1 = 0.5 * (tn + tn + dt - 2.0 * tm);
      c2 = 0.5 * (2.0 * tn - tn - dt - tm);
    }
    tau2 = dt + tn - tm;
  }
  const double kyr = k_full(a.ky0 + ky, a.ny_k ? a.ny_k : a.ny, a.ay);
  const double kzr = k_full(kz, a.nz, a.az);
  const bool need_u = a.bandlim || MODE != FIN_RHS;
  double esum = 0.0, dsum = 0.0;
  for (int kx0 = lane; kx0 < a.nxh; kx0 += 32 * CH) {
    C nn[CH][3], uu[CH][3], ss[CH][3], no[CH][3];
    bool ok[CH];
#pragma unroll
    for (int h = 0; h < CH; ++h) {
      const int kx = kx0 + 32 * h;
      ok[h] = kx < a.nxh && a.kx.keep(kx);
      const long long idx = rowbase + kx;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        nn[h][c] = ok[h] ? a.n3[c * n3nh + n3row + kx] : mkc<C>(0, 0);
        uu[h][c] = ok[h] && need_u ? a.uin[c * a.nh + idx] : mkc<C>(0, 0);
        ss[h][c] = ok[h] && MODE == FIN_CORR ? a.state[c * a.nh + idx] : mkc<C>(0, 0);
        no[h][c] = ok[h] && MODE == FIN_AB2 ? a.nold[c * a.nh + idx] : mkc<C>(0, 0);
      }
    }
#pragma unroll
    for (int h = 0; h < CH; ++h) {
      if (!ok[h]) continue;
      const int kx = kx0 + 32 * h;
      const long long idx = rowbase + kx;
      const double kxr = k_half(kx, a.nx, a.ax);
      const double wk = (kxr == 0.0) ? 0.5 : 1.0;   // state.f90:436-440
      const double k2 = kxr * kxr + kyr * kyr + kzr * kzr;
      const bool zero = (kxr == 0.0) && (kyr == 0.0) && (kzr == 0.0);
      const bool cut = (a.spherical && k2 >= a.sph2) || fabs(kxr) >= a.cutx || fabs(kyr) >= a.cuty ||
                       fabs(kzr) >= a.cutz || zero;
      C Nc[3];
      if (cut) {
        Nc[0] = Nc[1] = Nc[2] = mkc<C>(0, 0);
      } else {
        // phat = -(i k . n) / (-(k.k))  (rhs.f90:101-106), in T: the masks
        // above and below are decided in FP64 (the same kept set in every
        // precision), the pointwise arithmetic in the state's precision
        const T kr[3] = {T(kxr), T(kyr), T(kzr)}, k2t = T(k2);
        const T knre = kr[0] * nn[h][0].x + kr[1] * nn[h][1].x + kr[2] * nn[h][2].x;
        const T knim = kr[0] * nn[h][0].y + kr[1] * nn[h][1].y + kr[2] * nn[h][2].y;
        const T pre = -knim / k2t, pim = knre / k2t;
        const bool forced = a.bandlim && sqrt(k2) <= a.kcut;
        const T fct = T(fc);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          T re = -nn[h][c].x + kr[c] * pim;
          T im = -nn[h][c].y - kr[c] * pre;
          if (forced) {
            re += fct * uu[h][c].x;
            im += fct * uu[h][c].y;
          }
          if (a.force) {
            const C q = a.force[c * a.nh + idx];
            re += q.x;
            im += q.y;
          }
          Nc[c] = mkc<C>(re, im);
        }
      }
      if (MODE == FIN_RHS) {
#pragma unroll
        for (int c = 0; c < 3; ++c) a.out[c * a.nh + idx] = Nc[c];
        continue;
      }
      const T IF = if_exp<T>((a.Q - nu * k2) * dt);
      const T tdt = T(dt);
      if (MODE == FIN_PRED) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const C u = uu[h][c];
          a.out[c * a.nh + idx] = mkc<C>((u.x + tdt * Nc[c].x) * IF, (u.y + tdt * Nc[c].y) * IF);
          if (a.nold) a.nold[c * a.nh + idx] = Nc[c];
        }
        continue;
      }
      C un[3];
      if (MODE == FIN_CORR) {
        const T hf = T(0.5), hdt = T(0.5 * dt);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const C u = ss[h][c], us = uu[h][c];
          un[c] = mkc<C>(hf * (IF * u.x + us.x) + hdt * Nc[c].x, hf * (IF * u.y + us.y) + hdt * Nc[c].y);
          a.state[c * a.nh + idx] = un[c];
        }
      } else {  // FIN_AB2
        const T e1c1 = T(c1) * IF;
        const T e2c2 = T(c2) * if_exp<T>((a.Q - nu * k2) * tau2);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const C u = uu[h][c], o = no[h][c];
          un[c] = mkc<C>(IF * u.x + e1c1 * Nc[c].x + e2c2 * o.x, IF * u.y + e1c1 * Nc[c].y + e2c2 * o.y);
          a.state[c * a.nh + idx] = un[c];
          a.nold[c * a.nh + idx] = Nc[c];
        }
      }
      double e2 = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) e2 += (double)un[c].x * un[c].x + (double)un[c].y * un[c].y;
      esum += wk * e2;
      dsum += 2.0 * wk * k2 * e2;
    }
  }
  if (a.partials) {
    esum = warp_sum(esum);
    dsum = warp_sum(dsum);
    if (lane == 0) {
      double *pp = a.partials + 2 * ((long long)box * a.nz * a.ny + (long long)kz * a.ny + ky);
      pp[0] = esum;
      pp[1] = dsum;
    }
  }
}


}  // namespace dnsbox
