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
// max|u_i| (CFL) reduction and the first forward x pass (k_xline_nl); the last
// forward z pass is fused with dealiasing, pressure projection, band forcing,
// the integrating-factor stepper and the energy/dissipation reductions
// (k_zfinish).
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace dnsbox {

// Blocks are launched with a multiple of 32 threads (full warps for the
// shuffle reductions); threads beyond the FFT's own count only take part in
// the strided element loops and barriers.
__host__ __device__ constexpr int round32(int x) { return (x + 31) / 32 * 32; }

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
  int ks1, ks2;            // 0: kx of the column, 1: wavenumber of the row index
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
};

template <typename T, typename C>
__device__ __forceinline__ C apply_mult(C v, double a, double b, double k) {
  // v * (a + i b k)
  const T bk = T(b * k), aa = T(a);
  return mkc<C>(v.x * aa - v.y * bk, v.y * aa + v.x * bk);
}

template <typename T, int N, bool INV>
__global__ void __launch_bounds__(round32(TileCols<T>::v *(N / FftPlan<N>::E)))
    k_strided(const __grid_constant__ StridedArgs<T> a) {
  using C = typename CT<T>::type;
  constexpr int TC = TileCols<T>::v;
  constexpr int NF = TC * (N / FftPlan<N>::E);   // FFT threads
  const int NT = blockDim.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s = reinterpret_cast<C *>(smem_raw);
  const int job = blockIdx.x % a.njobs;
  const int tile = blockIdx.x / a.njobs;
  const int ntx = (a.ncols + TC - 1) / TC;
  const int other = tile / ntx;
  const int kx0 = (tile - other * ntx) * TC;
  const StridedJob<T> &J = a.job[job];
  const long long base = (long long)other * a.otherstride + kx0;
  const bool plain1 = (J.a1 == 1.0 && J.b1 == 0.0);
  for (int e = threadIdx.x; e < N * TC; e += NT) {
    const int row = e / TC, col = e - (e / TC) * TC;
    const int kx = kx0 + col;
    C v = mkc<C>(0, 0);
    if (kx < a.ncols) {
      const long long off = base + (long long)row * a.rowstride + col;
      v = J.in1[off];
      if (!plain1) {
        const double k = J.ks1 ? k_full(row, N, a.alpha_row) : k_half(kx, a.nx, a.alpha_x);
        v = apply_mult<T>(v, J.a1, J.b1, k);
      }
      if (J.in2) {
        const double k = J.ks2 ? k_full(row, N, a.alpha_row) : k_half(kx, a.nx, a.alpha_x);
        v = cadd(v, apply_mult<T>(J.in2[off], J.a2, J.b2, k));
      }
    }
    s[e] = v;
  }
  __syncthreads();
  const int col = threadIdx.x % TC, p = threadIdx.x / TC;
  fft_columns<C, N, INV>(s, TC, col, p, threadIdx.x < NF, a.tw);
  for (int e = threadIdx.x; e < N * TC; e += NT) {
    const int row = e / TC, col2 = e - (e / TC) * TC;
    if (kx0 + col2 < a.ncols) J.out[base + (long long)row * a.rowstride + col2] = s[e];
  }
}

// ------------------------------------------------------------------ x lines
template <typename T> struct XlineNLArgs {
  using C = typename CT<T>::type;
  const C *U, *V, *W, *OX, *B1, *C1;  // (kx, y, z) space, rows of nxh
  C *NX, *NY, *NZ;                     // forward x transforms of (omega x u) * s
  const C *tw;
  double *umax;                        // 3 values, max |u_i| (true scale)
  int nlines, nxh;
  double alpha_x;
  double s;                            // scalemodes
};

// Lines per CTA of the fused x pass (even; 3B columns in shared memory).
template <typename T, int N> struct XlineB {
  static constexpr int v = (N >= 512) ? 2 : (sizeof(T) == 8 ? (N >= 256 ? 4 : 8) : (N >= 256 ? 8 : 16));
};

template <typename T, int N>
__global__ void __launch_bounds__(round32(3 * XlineB<T, N>::v *(N / FftPlan<N>::E)))
    k_xline_nl(const __grid_constant__ XlineNLArgs<T> a) {
  using C = typename CT<T>::type;
  constexpr int B = XlineB<T, N>::v;
  constexpr int H = N / 2 + 1;
  constexpr int LD = 3 * B;
  constexpr int P = N / FftPlan<N>::E;
  constexpr int NF = 3 * B * P;        // FFT threads of the inverse transforms
  const int NT = blockDim.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s = reinterpret_cast<C *>(smem_raw);
  __shared__ double red[3 * 32];
  const int line0 = blockIdx.x * B;
  const T sc = T(a.s);
  // Build Z = X1 + i X2.  Each pair holds two quantities of the same kind and
  // scale (velocity is unscaled, vorticity carries the 1/N^3 of the
  // reference's derivative transforms), so neither loses bits to the other.
  // Per line pair (a = 2j, b = 2j+1) the six columns are
  //   (u_a, v_a) (u_b, v_b) (w_a, w_b) (ox_a, oy_a) (ox_b, oy_b) (oz_a, oz_b).
  for (int it = threadIdx.x; it < (B / 2) * 6 * H; it += NT) {
    const int k = it % H;
    const int q = (it / H) % 6;
    const int j = it / (6 * H);
    const int la = line0 + 2 * j, lb = la + 1;
    const int col = 6 * j + q;
    const T kx = T(k_half(k, N, a.alpha_x)) * sc;
    const long long oa = (long long)la * a.nxh + k, ob = (long long)lb * a.nxh + k;
    const bool va = la < a.nlines, vb = lb < a.nlines;
    C X1 = mkc<C>(0, 0), X2 = mkc<C>(0, 0);
    switch (q) {
      case 0:
        if (va) { X1 = a.U[oa]; X2 = a.V[oa]; }
        break;
      case 1:
        if (vb) { X1 = a.U[ob]; X2 = a.V[ob]; }
        break;
      case 2:
        if (va) X1 = a.W[oa];
        if (vb) X2 = a.W[ob];
        break;
      case 3:
      case 4: {
        // omega_x, and omega_y = dz u - dx w (kx still spectral here)
        const bool v = q == 3 ? va : vb;
        const long long o = q == 3 ? oa : ob;
        if (v) {
          const C w = a.W[o], b1 = a.B1[o];
          X1 = a.OX[o];
          X2 = mkc<C>(b1.x + kx * w.y, b1.y - kx * w.x);   // b1 - i kx s w
        }
        break;
      }
      default: {
        // omega_z = dx v - dy u for both lines
        if (va) {
          const C v = a.V[oa], c1 = a.C1[oa];
          X1 = mkc<C>(c1.x - kx * v.y, c1.y + kx * v.x);   // c1 + i kx s v
        }
        if (vb) {
          const C v = a.V[ob], c1 = a.C1[ob];
          X2 = mkc<C>(c1.x - kx * v.y, c1.y + kx * v.x);
        }
        break;
      }
    }
    if (k == 0 || k == N / 2) {
      s[k * LD + col] = mkc<C>(X1.x, X2.x);
    } else {
      s[k * LD + col] = mkc<C>(X1.x - X2.y, X1.y + X2.x);
      s[(N - k) * LD + col] = mkc<C>(X1.x + X2.y, X2.x - X1.y);
    }
  }
  __syncthreads();
  {
    const int col = threadIdx.x % (3 * B), p = threadIdx.x / (3 * B);
    fft_columns<C, N, true>(s, LD, col, p, threadIdx.x < NF, a.tw);
  }
  // products (omega x u) * s, written back as three complex sequences per
  // line pair: (px_a, py_a), (pz_a, pz_b), (px_b, py_b)
  double m0 = 0, m1 = 0, m2 = 0;
  for (int it = threadIdx.x; it < N * (B / 2); it += NT) {
    const int j = it % (B / 2), n = it / (B / 2);
    C *r = s + n * LD + 6 * j;
    T px[2], py[2], pz[2];
    const C c0 = r[0], c1 = r[1], c2 = r[2], c3 = r[3], c4 = r[4], c5 = r[5];
    const T uu[2] = {c0.x, c1.x}, vv[2] = {c0.y, c1.y}, ww[2] = {c2.x, c2.y};
    const T ox[2] = {c3.x, c4.x}, oy[2] = {c3.y, c4.y}, oz[2] = {c5.x, c5.y};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const T u = uu[h], v = vv[h], w = ww[h];
      px[h] = (oy[h] * w - oz[h] * v) * sc;
      py[h] = (oz[h] * u - ox[h] * w) * sc;
      pz[h] = (ox[h] * v - oy[h] * u) * sc;
      m0 = fmax(m0, fabs((double)u));
      m1 = fmax(m1, fabs((double)v));
      m2 = fmax(m2, fabs((double)w));
    }
    r[0] = mkc<C>(px[0], py[0]);
    r[1] = mkc<C>(pz[0], pz[1]);
    r[2] = mkc<C>(px[1], py[1]);
  }
  __syncthreads();
  {
    constexpr int NQ = 3 * B / 2;
    const bool active = threadIdx.x < NQ * P;
    const int q = threadIdx.x % NQ, p = threadIdx.x / NQ;
    const int col = 6 * (q / 3) + q % 3;
    fft_columns<C, N, false>(s, LD, col, p, active, a.tw);
  }
  // unpack two real transforms per sequence and store
  for (int it = threadIdx.x; it < (3 * B / 2) * H; it += NT) {
    const int k = it % H, q = it / H;
    const int j = q / 3, c = q % 3;
    const int col = 6 * j + c;
    const C zk = s[k * LD + col], zn = s[((N - k) % N) * LD + col];
    const C X1 = mkc<C>(T(0.5) * (zk.x + zn.x), T(0.5) * (zk.y - zn.y));
    const C X2 = mkc<C>(T(0.5) * (zk.y + zn.y), T(-0.5) * (zk.x - zn.x));
    const int la = line0 + 2 * j, lb = la + 1;
    if (c == 0) {
      if (la < a.nlines) {
        a.NX[(long long)la * a.nxh + k] = X1;
        a.NY[(long long)la * a.nxh + k] = X2;
      }
    } else if (c == 1) {
      if (la < a.nlines) a.NZ[(long long)la * a.nxh + k] = X1;
      if (lb < a.nlines) a.NZ[(long long)lb * a.nxh + k] = X2;
    } else {
      if (lb < a.nlines) {
        a.NX[(long long)lb * a.nxh + k] = X1;
        a.NY[(long long)lb * a.nxh + k] = X2;
      }
    }
  }
  // CFL reduction
  m0 = warp_max(m0);
  m1 = warp_max(m1);
  m2 = warp_max(m2);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[wid] = m0;
    red[32 + wid] = m1;
    red[64 + wid] = m2;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = NT >> 5;
    double x0 = lane < nw ? red[lane] : 0, x1 = lane < nw ? red[32 + lane] : 0,
           x2 = lane < nw ? red[64 + lane] : 0;
    x0 = warp_max(x0);
    x1 = warp_max(x1);
    x2 = warp_max(x2);
    if (lane == 0 && a.umax) {
      atomic_max_nonneg(a.umax + 0, x0 * a.s);
      atomic_max_nonneg(a.umax + 1, x1 * a.s);
      atomic_max_nonneg(a.umax + 2, x2 * a.s);
    }
  }
}

// Plain x-line transforms of nf fields (blockIdx.y = field).
template <typename T> struct XlineArgs {
  using C = typename CT<T>::type;
  const void *in[3];
  void *out[3];
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
  constexpr int B = XlinePlainB<T, N>::v;
  constexpr int NC = B / 2;
  constexpr int H = N / 2 + 1;
  constexpr int NF = NC * (N / FftPlan<N>::E);
  const int NT = blockDim.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s = reinterpret_cast<C *>(smem_raw);
  const C *in = reinterpret_cast<const C *>(a.in[blockIdx.y]);
  T *out = reinterpret_cast<T *>(a.out[blockIdx.y]);
  const int line0 = blockIdx.x * B;
  for (int it = threadIdx.x; it < NC * H; it += NT) {
    const int k = it % H, j = it / H;
    const int la = line0 + 2 * j, lb = la + 1;
    const C X1 = la < a.nlines ? in[(long long)la * a.nxh + k] : mkc<C>(0, 0);
    const C X2 = lb < a.nlines ? in[(long long)lb * a.nxh + k] : mkc<C>(0, 0);
    if (k == 0 || k == N / 2) {
      s[k * NC + j] = mkc<C>(X1.x, X2.x);
    } else {
      s[k * NC + j] = mkc<C>(X1.x - X2.y, X1.y + X2.x);
      s[(N - k) * NC + j] = mkc<C>(X1.x + X2.y, X2.x - X1.y);
    }
  }
  __syncthreads();
  fft_columns<C, N, true>(s, NC, threadIdx.x % NC, threadIdx.x / NC, threadIdx.x < NF, a.tw);
  const T sc = T(a.scale);
  for (int it = threadIdx.x; it < NC * N; it += NT) {
    const int n = it % N, j = it / N;
    const int la = line0 + 2 * j, lb = la + 1;
    const C z = s[n * NC + j];
    if (la < a.nlines) out[(long long)la * N + n] = z.x * sc;
    if (lb < a.nlines) out[(long long)lb * N + n] = z.y * sc;
  }
}

// R2C along x: real lines -> half lines, two lines per FFT.
template <typename T, int N>
__global__ void __launch_bounds__(round32((XlinePlainB<T, N>::v / 2) * (N / FftPlan<N>::E)))
    k_xline_r2c(const __grid_constant__ XlineArgs<T> a) {
  using C = typename CT<T>::type;
  constexpr int B = XlinePlainB<T, N>::v;
  constexpr int NC = B / 2;
  constexpr int H = N / 2 + 1;
  constexpr int NF = NC * (N / FftPlan<N>::E);
  const int NT = blockDim.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s = reinterpret_cast<C *>(smem_raw);
  const T *in = reinterpret_cast<const T *>(a.in[blockIdx.y]);
  C *out = reinterpret_cast<C *>(a.out[blockIdx.y]);
  const int line0 = blockIdx.x * B;
  for (int it = threadIdx.x; it < NC * N; it += NT) {
    const int n = it % N, j = it / N;
    const int la = line0 + 2 * j, lb = la + 1;
    const T x1 = la < a.nlines ? in[(long long)la * N + n] : T(0);
    const T x2 = lb < a.nlines ? in[(long long)lb * N + n] : T(0);
    s[n * NC + j] = mkc<C>(x1, x2);
  }
  __syncthreads();
  fft_columns<C, N, false>(s, NC, threadIdx.x % NC, threadIdx.x / NC, threadIdx.x < NF, a.tw);
  const T sc = T(a.scale);
  for (int it = threadIdx.x; it < NC * H; it += NT) {
    const int k = it % H, j = it / H;
    const int la = line0 + 2 * j, lb = la + 1;
    const C zk = s[k * NC + j], zn = s[((N - k) % N) * NC + j];
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
  const C *n3;             // 3 fields (kx, ky, z) after the forward y pass
  const C *uin;            // 3 fields, RHS input (forcing)
  C *out;                  // FIN_RHS / FIN_PRED output (3 fields)
  C *state;                // FIN_CORR state (3 fields)
  C *nold;                 // AB2 history (3 fields)
  const StepState *st;
  double *partials;        // per-CTA (E, D) of the new state, or null
  const C *tw;
  long long nh;            // elements per field
  int nx, ny, nz, nxh;
  double ax, ay, az;
  double nu, Q, Pin, kcut;
  double cutx, cuty, cutz, sph2;
  int bandlim, spherical, mode, ab2_standard;
  double s;                // scalemodes
};

template <typename T, int N>
__global__ void __launch_bounds__(round32(TileCols<T>::v *(N / FftPlan<N>::E)))
    k_zfinish(const __grid_constant__ FinishArgs<T> a) {
  using C = typename CT<T>::type;
  constexpr int TC = TileCols<T>::v;
  constexpr int NF = TC * (N / FftPlan<N>::E);
  const int NT = blockDim.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s = reinterpret_cast<C *>(smem_raw);
  __shared__ double red[2 * 32];
  const int ntx = (a.nxh + TC - 1) / TC;
  const int ky = blockIdx.x / ntx;
  const int kx0 = (blockIdx.x - ky * ntx) * TC;
  const long long rowstride = (long long)a.ny * a.nxh;
  const long long base = (long long)ky * a.nxh + kx0;
  for (int f = 0; f < 3; ++f) {
    const C *src = a.n3 + f * a.nh;
    for (int e = threadIdx.x; e < N * TC; e += NT) {
      const int row = e / TC, col = e - (e / TC) * TC;
      s[f * N * TC + e] = (kx0 + col < a.nxh) ? src[base + row * rowstride + col] : mkc<C>(0, 0);
    }
  }
  __syncthreads();
  const int col = threadIdx.x % TC, p = threadIdx.x / TC;
  for (int f = 0; f < 3; ++f) fft_columns<C, N, false>(s + f * N * TC, TC, col, p, threadIdx.x < NF, a.tw);

  const StepState *st = a.st;
  const double dt = st ? st->dt : 0.0;
  const double fc = (a.bandlim && st) ? a.Pin / (2.0 * st->eband) : 0.0;
  double c1 = 0, c2 = 0, tau2 = 0;
  if (a.mode == FIN_AB2) {
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
  const double kyr = k_full(ky, a.ny, a.ay);
  double esum = 0.0, dsum = 0.0;
  for (int e = threadIdx.x; e < N * TC; e += NT) {
    const int kz = e / TC, cl = e - (e / TC) * TC;
    const int kx = kx0 + cl;
    if (kx >= a.nxh) continue;
    const long long idx = (long long)kz * rowstride + base + cl;
    const double kxr = k_half(kx, a.nx, a.ax), kzr = k_full(kz, N, a.az);
    const double k2 = kxr * kxr + kyr * kyr + kzr * kzr;
    const bool zero = (kxr == 0.0) && (kyr == 0.0) && (kzr == 0.0);
    const bool cut = (a.spherical && k2 >= a.sph2) || fabs(kxr) >= a.cutx || fabs(kyr) >= a.cuty ||
                     fabs(kzr) >= a.cutz || zero;
    C Nc[3];
    if (cut) {
      Nc[0] = Nc[1] = Nc[2] = mkc<C>(0, 0);
    } else {
      const C n0 = s[e], n1 = s[N * TC + e], n2 = s[2 * N * TC + e];
      // phat = -(i k . n) / (-(k.k))  (rhs.f90:101-106)
      const double knre = kxr * (double)n0.x + kyr * (double)n1.x + kzr * (double)n2.x;
      const double knim = kxr * (double)n0.y + kyr * (double)n1.y + kzr * (double)n2.y;
      const double pre = -knim / k2, pim = knre / k2;
      const double kr[3] = {kxr, kyr, kzr};
      const C nn[3] = {n0, n1, n2};
      const bool forced = a.bandlim && sqrt(k2) <= a.kcut;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double re = -(double)nn[c].x + kr[c] * pim;
        double im = -(double)nn[c].y - kr[c] * pre;
        if (forced) {
          const C u = a.uin[c * a.nh + idx];
          re += fc * (double)u.x;
          im += fc * (double)u.y;
        }
        Nc[c] = mkc<C>(T(re), T(im));
      }
    }
    if (a.mode == FIN_RHS) {
#pragma unroll
      for (int c = 0; c < 3; ++c) a.out[c * a.nh + idx] = Nc[c];
      continue;
    }
    const T IF = T(exp((a.Q - a.nu * k2) * dt));
    const T tdt = T(dt);
    if (a.mode == FIN_PRED) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const C u = a.uin[c * a.nh + idx];
        a.out[c * a.nh + idx] = mkc<C>((u.x + tdt * Nc[c].x) * IF, (u.y + tdt * Nc[c].y) * IF);
        if (a.nold) a.nold[c * a.nh + idx] = Nc[c];
      }
      continue;
    }
    C un[3];
    if (a.mode == FIN_CORR) {
      const T h = T(0.5), hdt = T(0.5 * dt);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const C u = a.state[c * a.nh + idx], us = a.uin[c * a.nh + idx];
        un[c] = mkc<C>(h * (IF * u.x + us.x) + hdt * Nc[c].x, h * (IF * u.y + us.y) + hdt * Nc[c].y);
        a.state[c * a.nh + idx] = un[c];
      }
    } else {  // FIN_AB2
      const T e1c1 = T(c1) * IF;
      const T e2c2 = T(c2 * exp((a.Q - a.nu * k2) * tau2));
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const C u = a.uin[c * a.nh + idx], no = a.nold[c * a.nh + idx];
        un[c] = mkc<C>(IF * u.x + e1c1 * Nc[c].x + e2c2 * no.x, IF * u.y + e1c1 * Nc[c].y + e2c2 * no.y);
        a.state[c * a.nh + idx] = un[c];
        a.nold[c * a.nh + idx] = Nc[c];
      }
    }
    if (a.partials) {
      const double wk = (kxr == 0.0) ? 0.5 : 1.0;   // state.f90:436-440
      double e2 = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) e2 += (double)un[c].x * un[c].x + (double)un[c].y * un[c].y;
      esum += wk * e2;
      dsum += 2.0 * wk * k2 * e2;
    }
  }
  if (a.partials) {
    double v[2] = {esum, dsum};
    block_sum<2>(v, red);
    if (threadIdx.x == 0) {
      a.partials[2 * blockIdx.x] = v[0];
      a.partials[2 * blockIdx.x + 1] = v[1];
    }
  }
}

}  // namespace dnsbox
