// C ABI of libdnsbox_gpu.so: context, buffers, step orchestration and the
// small reduction / layout kernels.  See include/dnsbox.h for the contract.
//
// One right-hand side (rhs_nonlinear, rhs.f90:18-135) is five passes over HBM:
//   A  inverse z FFT of u, v, w, -dz v, dz u          (3 fields in, 5 out)
//   B  inverse y FFT, forming omega_x, dz u, -dy u     (5 in, 6 out)
//   C  inverse x C2R, (omega x u)*s, max|u_i|, forward x R2C  (6 in, 3 out)
//   D  forward y FFT                                   (3 in, 3 out)
//   E  forward z FFT + dealias + projection + forcing + stepper + E/D sums
// instead of the reference's 15 p3dfft transforms plus pointwise loops.
#include <cudaTypedefs.h>

#include <mutex>

#include "internal.cuh"

static thread_local std::string g_last_error;

int set_err(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}
static const int kSizes[] = {8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 512, 1024};

extern "C" int dnsbox_supported_size(int n) {
  for (int s : kSizes)
    if (s == n) return 1;
  return 0;
}

extern "C" int dnsbox_abi_version(void) { return DNSBOX_ABI_VERSION; }
extern "C" const char *dnsbox_last_error(void) { return g_last_error.c_str(); }

extern "C" void dnsbox_default_params(dnsbox_params *p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  // parameters.f90:11-50
  p->nx = p->ny = p->nz = 128;
  p->precision = DNSBOX_FP64;
  p->stepper = DNSBOX_HEUN;
  p->ab2_mode = DNSBOX_AB2_REFERENCE;
  p->bandlim = 1;
  p->spherical = 0;
  p->tstep_fix = 0;
  p->hminone = 1;
  p->spectrum_mode = DNSBOX_SPECTRUM_MPI;
  p->adj_phat = DNSBOX_ADJ_PHAT_INTENT;
  p->alpha_x = p->alpha_y = p->alpha_z = 1.0;
  p->nu = 0.005;
  p->Q = 0.0;
  p->kCutOff = 2.0;
  p->Pin = 0.1;
  p->Deltak = 1.0;
  p->courant_min = 0.15;
  p->courant_max = 0.2;
  p->dt_max = 1.0e-2;
  p->dt = 1.0e-3;   // variables.f90:9
  p->implicit_c = 0.5;          // parameters.f90:47
  p->implicit_tol = 1.0e-10;    // parameters.f90:26
  p->implicit_max_iter = 50;
}

// ------------------------------------------------------------ small kernels
// io_Courant (io.f90:664-676) on the fused max|u_i| and, when control is on,
// set_time_step (dnsboxheun.f90:153-157, 227-246).
__global__ void k_cfl(StepState *sts, int nbatch, double dx, double dy, double dz, int control, int force,
                      double cmin, double cmax, double dtmax, dnsbox_diag *ring, int ring_cap) {
  const int box = blockIdx.x * blockDim.x + threadIdx.x;
  if (box >= nbatch) return;
  StepState *st = sts + box;
  dnsbox_diag *drec = ring ? ring + ((long long)st->step % ring_cap) * nbatch + box : nullptr;
  double dt = st->dt;
  double C = st->umax[0] * dt / dx + st->umax[1] * dt / dy + st->umax[2] * dt / dz;
  if (control && (force || C > cmax || (C < cmin && dt < dtmax))) {
    double nd = ((cmax + cmin) / (2.0 * C)) * dt;
    if (nd > dtmax) nd = dtmax;
    C = C * nd / dt;
    st->dt = nd;
    dt = nd;
  }
  st->courant = C;
  st->eband1 = st->eband;
  if (drec) {
    drec->courant = C;
    drec->umax[0] = st->umax[0];
    drec->umax[1] = st->umax[1];
    drec->umax[2] = st->umax[2];
    drec->eband = st->eband;
    drec->dt = dt;
  }
}

// Sums the finish-kernel partials (fixed order), writes the step record and
// advances the clock.
// Per-plane sums of the spectral finish's row partials: block (kz, box) adds
// the (E, D) pairs of the ny rows of plane kz in a fixed order.  Rows and
// planes outside the kept ky / kz sets of a pruned step were not visited and
// count as zero.
__global__ void k_plane_sums(const double *rows, double *planes, int nz, int ny, AxisKeep ky, AxisKeep kz) {
  __shared__ double red[2 * 32];
  const int iz = blockIdx.x, box = blockIdx.y;
  const double *r = rows + 2 * ((long long)box * nz + iz) * ny;
  double e = 0.0, d = 0.0;
  if (kz.keep(iz))
    for (int j = threadIdx.x; j < ny; j += blockDim.x)
      if (ky.keep(j)) {
        e += r[2 * j];
        d += r[2 * j + 1];
      }
  double v[2] = {e, d};
  block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    planes[2 * ((long long)box * nz + iz)] = v[0];
    planes[2 * ((long long)box * nz + iz) + 1] = v[1];
  }
}

// one block per box; partials: np (E, D) pairs per box (the plane sums)
__global__ void k_finalize(StepState *sts, const double *partials, int np, double s2, double nu,
                           const double *nu_box, double Q, double Pin, int bandlim, dnsbox_diag *ring,
                           int ring_cap) {
  __shared__ double red[2 * 32];
  const int box = blockIdx.x, nbatch = gridDim.x;
  StepState *st = sts + box;
  partials += 2 * (long long)box * np;
  if (nu_box) nu = nu_box[box];
  dnsbox_diag *drec = ring ? ring + ((long long)st->step % ring_cap) * nbatch + box : nullptr;
  double e = 0.0, d = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    e += partials[2 * i];
    d += partials[2 * i + 1];
  }
  double v[2] = {e, d};
  block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    const double E = v[0] * s2, D = nu * v[1] * s2;
    const double dt = st->dt;
    if (drec) {
      drec->t = st->t + dt;
      drec->dt = dt;
      drec->ekin = E;
      drec->dissipation = D;
      drec->production_literal = 2.0 * Q * E;
      drec->injected_power = (bandlim ? Pin : 0.0) + 2.0 * Q * E;
      drec->nonfinite = !(isfinite(E) && isfinite(D));
      drec->step = (int)st->step + 1;
    }
    st->t_prev = st->t;
    st->t = st->t + dt;
    st->step += 1.0;
  }
}

__global__ void k_reset_umax(StepState *st, int nbatch) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nbatch) st[b].umax[0] = st[b].umax[1] = st[b].umax[2] = 0.0;
}

// sets the double at byte offset `off` of every box's StepState
__global__ void k_set_state(StepState *st, int nbatch, int off, double v) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nbatch) *reinterpret_cast<double *>(reinterpret_cast<char *>(st + b) + off) = v;
}

// Spectral diagnostics over the half spectrum: shell spectrum (state.f90:350-411
// or single/state.f90:191-230), EZero/EOne/Esqrt2, kinetic energy
// (state.f90:429-454) and the Parseval dissipation sum.  Per-block partials
// [gridDim][NV], NV = nspec + 5.
template <typename C>
__global__ void k_specdiag(const C *u, long long nh, int nx, int ny, int nz, double ax, double ay,
                           double az, int nspec, double deltak, int single, double s2,
                           double *partials) {
  extern __shared__ double hist[];
  const int NV = nspec + 5;
  for (int i = threadIdx.x; i < NV; i += blockDim.x) hist[i] = 0.0;
  __syncthreads();
  const int nxh = nx / 2 + 1;
  const double sq2 = sqrt(2.0);
  double ez = 0, e1 = 0, es = 0, ek = 0, dk = 0;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < nh;
       m += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(m % nxh);
    const int ky = (int)((m / nxh) % ny);
    const int kz = (int)(m / ((long long)nxh * ny));
    const double kxr = k_half(kx, nx, ax), kyr = k_full(ky, ny, ay), kzr = k_full(kz, nz, az);
    const double k2 = kxr * kxr + kyr * kyr + kzr * kzr;
    const double absk = sqrt(k2);
    double e2 = 0.0;
    for (int c = 0; c < 3; ++c) {
      const C v = u[c * nh + m];
      e2 += (double)v.x * v.x + (double)v.y * v.y;
    }
    const double w = (kxr == 0.0) ? 0.5 : 1.0;
    ek += w * e2;
    dk += 2.0 * w * k2 * e2;
    const double base = floor(absk / deltak);
    const int nk = (absk < base + 0.5 * deltak) ? (int)base : (int)base + 1;
    if (!single) {
      if (absk == 0.0) ez += e2;
      if (absk == 1.0) e1 += e2;
      if (absk - sq2 < 1.0e-9) es += e2;
      if (nk < nspec && nk != 0) atomicAdd(&hist[nk - 1], e2 * s2 / deltak);
    } else {
      if (absk == 0.0) ez += w * e2;
      if (nk <= nspec && nk != 0) atomicAdd(&hist[nk - 1], w * e2 * s2 / deltak);
    }
  }
  __shared__ double red[5 * 32];
  double v[5] = {ez, e1, es, ek, dk};
  block_sum<5>(v, red);
  if (threadIdx.x == 0)
    for (int i = 0; i < 5; ++i) hist[nspec + i] = v[i];
  __syncthreads();
  for (int i = threadIdx.x; i < NV; i += blockDim.x) partials[(long long)blockIdx.x * NV + i] = hist[i];
}

__global__ void k_sum_partials(const double *partials, int nblk, int nv, double *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += partials[(long long)b * nv + i];
    out[i] = s;
  }
}

// max (signed or |.|) of a real array: per-block partials
template <typename T>
__global__ void k_max(const T *f, long long n, int absval, double *partials) {
  __shared__ double red[32];
  double m = -INFINITY;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double x = (double)f[i];
    m = fmax(m, absval ? fabs(x) : x);
  }
  m = warp_max(m);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = m;
  __syncthreads();
  if (wid == 0) {
    double x = lane < (int)(blockDim.x >> 5) ? red[lane] : -INFINITY;
    x = warp_max(x);
    if (lane == 0) partials[blockIdx.x] = x;
  }
}

__global__ void k_max_partials(const double *partials, int nblk, double *out) {
  __shared__ double red[32];
  double m = -INFINITY;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) m = fmax(m, partials[i]);
  m = warp_max(m);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = m;
  __syncthreads();
  if (wid == 0) {
    double x = lane < (int)(blockDim.x >> 5) ? red[lane] : -INFINITY;
    x = warp_max(x);
    if (lane == 0) *out = x;
  }
}

// state_project (state.f90:120-179), in place
template <typename C>
__global__ void k_project(C *u, long long nh, int nx, int ny, int nz, double ax, double ay, double az) {
  using T = decltype(C{}.x);
  const int nxh = nx / 2 + 1;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < nh;
       m += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(m % nxh), ky = (int)((m / nxh) % ny), kz = (int)(m / ((long long)nxh * ny));
    const double kr[3] = {k_half(kx, nx, ax), k_full(ky, ny, ay), k_full(kz, nz, az)};
    if (kr[0] == 0.0 && kr[1] == 0.0 && kr[2] == 0.0) continue;
    const double k2 = kr[0] * kr[0] + kr[1] * kr[1] + kr[2] * kr[2];
    const C v[3] = {u[m], u[nh + m], u[2 * nh + m]};
    for (int i = 0; i < 3; ++i) {
      double re = v[i].x, im = v[i].y;
      for (int j = 0; j < 3; ++j) {
        re -= (kr[i] * kr[j] * (double)v[j].x) / k2;
        im -= (kr[i] * kr[j] * (double)v[j].y) / k2;
      }
      u[i * nh + m] = mkc<C>(T(re), T(im));
    }
  }
}

// One fixed-point update of the semi-implicit step (dnsboximplicit.f90:112-173
// with rhsFix / rhstStepFact restated as the theta scheme of nsbox.f90:192-221):
//   fac = 1 / (1/dt - c L),  fix = (1/dt + (1 - c) L) u_n,  L = Q - nu |k|^2
//   FIRST: u = fac (fix + n0);  else u <- fac (fix + c nk + (1 - c) n0)
// and, for the iterations, chg[i] = max over the modes of |u_i new - u_i old|
// (block maxima, then an atomic maximum).  dt is the step's device-side dt.
template <typename C, bool FIRST>
__global__ void k_si_update(C *u, const C *un, const C *n0, const C *nk, long long nh, int nx, int ny, int nz,
                            double ax, double ay, double az, double nu, double Q, double cimp, const StepState *st,
                            double *chg) {
  using T = decltype(C{}.x);
  __shared__ double red[3 * 32];
  const int nxh = nx / 2 + 1;
  const double dt = st->dt;
  double mx[3] = {0.0, 0.0, 0.0};
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < nh;
       m += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(m % nxh), ky = (int)((m / nxh) % ny), kz = (int)(m / ((long long)nxh * ny));
    const double kxr = k_half(kx, nx, ax), kyr = k_full(ky, ny, ay), kzr = k_full(kz, nz, az);
    const double L = Q - nu * (kxr * kxr + kyr * kyr + kzr * kzr);
    const double fac = 1.0 / (1.0 / dt - cimp * L), g = 1.0 / dt + (1.0 - cimp) * L;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const long long q = i * nh + m;
      const C a = un[q], b = n0[q];
      double re, im;
      if (FIRST) {
        re = fac * (g * (double)a.x + (double)b.x);
        im = fac * (g * (double)a.y + (double)b.y);
      } else {
        const C d = nk[q], o = u[q];
        re = fac * (g * (double)a.x + cimp * (double)d.x + (1.0 - cimp) * (double)b.x);
        im = fac * (g * (double)a.y + cimp * (double)d.y + (1.0 - cimp) * (double)b.y);
        const C w = mkc<C>(T(re), T(im));
        mx[i] = fmax(mx[i], hypot((double)w.x - (double)o.x, (double)w.y - (double)o.y));
      }
      u[q] = mkc<C>(T(re), T(im));
    }
  }
  if (FIRST) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 3; ++i) mx[i] = warp_max(mx[i]);
  if (lane == 0)
    for (int i = 0; i < 3; ++i) red[32 * i + wid] = mx[i];
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    for (int i = 0; i < 3; ++i) {
      const double x = warp_max(lane < nw ? red[32 * i + lane] : 0.0);
      if (lane == 0) atomic_max_nonneg(chg + i, x);
    }
  }
}

// Per-(kz, ky) row sums of E and D of a state (the partials the spectral
// finish writes for the Heun and AB2 steps), one warp per row, fixed order.
template <typename C>
__global__ void k_row_sums(const C *u, long long nh, long long fstride, int nx, int ny, int nz, double ax,
                           double ay, double az, double *partials) {
  const int nxh = nx / 2 + 1;
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= ny * nz) return;
  u += (long long)blockIdx.y * nh;   // box blockIdx.y; components fstride apart
  partials += 2 * (long long)blockIdx.y * nz * ny;
  const int kz = w / ny, ky = w - kz * ny;
  const double kyr = k_full(ky, ny, ay), kzr = k_full(kz, nz, az);
  const long long row = (long long)w * nxh;
  double es = 0.0, ds = 0.0;
  for (int kx = lane; kx < nxh; kx += 32) {
    const double kxr = k_half(kx, nx, ax);
    const double wk = kxr == 0.0 ? 0.5 : 1.0, k2 = kxr * kxr + kyr * kyr + kzr * kzr;
    double e2 = 0.0;
    for (int i = 0; i < 3; ++i) {
      const C v = u[i * fstride + row + kx];
      e2 += (double)v.x * v.x + (double)v.y * v.y;
    }
    es += wk * e2;
    ds += 2.0 * wk * k2 * e2;
  }
  es = warp_sum(es);
  ds = warp_sum(ds);
  if (lane == 0) {
    partials[2 * (long long)w] = es;
    partials[2 * (long long)w + 1] = ds;
  }
}

// Uniform noise in [-0.5, 0.5) from a counter-based hash of (seed, index)
// (SplitMix64 finaliser; Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014).
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
template <typename T> __global__ void k_noise(T *out, long long n, uint64_t seed) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const uint64_t h = splitmix64(seed * 0xD1B54A32D192ED03ull + (uint64_t)i);
    out[i] = (T)((double)(h >> 11) * 0x1.0p-53 - 0.5);
  }
}

// state_init_analytic (state.f90:287-307): the Beltrami (Shapiro) field at
// time t on the grid x(i) = i Lx / Nx, i = -Nx/2 .. Nx/2 - 1
// (variables.f90:235-266); physical [3][z][y][x].
template <typename T>
__global__ void k_beltrami(T *u, int nx, int ny, int nz, double lx, double ly, double lz, double nu, double t) {
  const long long np = (long long)nx * ny * nz;
  const double f = sqrt(3.0), dec = exp(-(f * f) * t * nu);
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < np;
       m += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(m % nx), iy = (int)((m / nx) % ny), iz = (int)(m / ((long long)nx * ny));
    const double x = (ix - nx / 2) * lx / nx, y = (iy - ny / 2) * ly / ny, z = (iz - nz / 2) * lz / nz;
    u[m] = (T)(-0.5 * (f * cos(x) * sin(y) * sin(z) + sin(x) * cos(y) * cos(z)) * dec);
    u[np + m] = (T)(0.5 * (f * sin(x) * cos(y) * sin(z) - cos(x) * sin(y) * cos(z)) * dec);
    u[2 * np + m] = (T)(cos(x) * cos(y) * sin(z) * dec);
  }
}

// Shell rescale of state_init_rand (state.f90:256-283): the nearest window
// nk of |k| (the rounding of state.f90:363-367); modes with nk = 0 or
// nk >= nspec are zeroed, the others multiplied by
// sqrt(C1 (nk dk)^C2 exp(-C3 (nk dk)^C4) / espec[nk - 1]).
template <typename C>
__global__ void k_yoffe_rescale(C *u, long long nh, int nx, int ny, int nz, double ax, double ay, double az,
                                double dk, int nspec, const double *espec) {
  using T = decltype(C{}.x);
  const double c1 = 8.0e-2, c2 = 2.0, c3 = 8.2352309e-2, c4 = 2.0;   // state.f90:218-221
  const int nxh = nx / 2 + 1;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < nh;
       m += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(m % nxh), ky = (int)((m / nxh) % ny), kz = (int)(m / ((long long)nxh * ny));
    const double kxr = k_half(kx, nx, ax), kyr = k_full(ky, ny, ay), kzr = k_full(kz, nz, az);
    const double absk = sqrt(kxr * kxr + kyr * kyr + kzr * kzr);
    const double base = floor(absk / dk);
    const int nk = absk < base + 0.5 * dk ? (int)base : (int)base + 1;
    double f = 0.0;
    if (nk != 0 && nk < nspec) {
      const double kn = nk * dk;
      f = sqrt(c1 * pow(kn, c2) * exp(-c3 * pow(kn, c4)) / espec[nk - 1]);
    }
    for (int i = 0; i < 3; ++i) {
      const C v = u[i * nh + m];
      u[i * nh + m] = mkc<C>(T(v.x * f), T(v.y * f));
    }
  }
}

// state_project + state_dealias of every box (dnsboxband.f90:142-143): boxes
// on gridDim.y, components fstride apart, boxes nh apart.
template <typename C>
__global__ void k_project_dealias(C *u, long long nh, long long fstride, int nx, int ny, int nz, double ax,
                                  double ay, double az, int spherical, double cx, double cy, double cz, double sph2) {
  using T = decltype(C{}.x);
  const int nxh = nx / 2 + 1;
  u += (long long)blockIdx.y * nh;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < nh;
       m += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(m % nxh), ky = (int)((m / nxh) % ny), kz = (int)(m / ((long long)nxh * ny));
    const double kr[3] = {k_half(kx, nx, ax), k_full(ky, ny, ay), k_full(kz, nz, az)};
    const double k2 = kr[0] * kr[0] + kr[1] * kr[1] + kr[2] * kr[2];
    const bool zero = kr[0] == 0.0 && kr[1] == 0.0 && kr[2] == 0.0;
    const bool cut = (spherical && k2 >= sph2) || fabs(kr[0]) >= cx || fabs(kr[1]) >= cy || fabs(kr[2]) >= cz || zero;
    if (cut) {
      for (int i = 0; i < 3; ++i) u[i * fstride + m] = mkc<C>(0, 0);
      continue;
    }
    const C v[3] = {u[m], u[fstride + m], u[2 * fstride + m]};
    for (int i = 0; i < 3; ++i) {
      double re = v[i].x, im = v[i].y;
      for (int j = 0; j < 3; ++j) {
        re -= (kr[i] * kr[j] * (double)v[j].x) / k2;
        im -= (kr[i] * kr[j] * (double)v[j].y) / k2;
      }
      u[i * fstride + m] = mkc<C>(T(re), T(im));
    }
  }
}

// state_dealias (state.f90:181-209), in place
template <typename C>
__global__ void k_dealias(C *u, long long nh, int nx, int ny, int nz, double ax, double ay, double az,
                          int spherical, double cx, double cy, double cz, double sph2) {
  const int nxh = nx / 2 + 1;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < nh;
       m += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(m % nxh), ky = (int)((m / nxh) % ny), kz = (int)(m / ((long long)nxh * ny));
    const double kxr = k_half(kx, nx, ax), kyr = k_full(ky, ny, ay), kzr = k_full(kz, nz, az);
    const double k2 = kxr * kxr + kyr * kyr + kzr * kzr;
    const bool cut = (spherical && k2 >= sph2) || fabs(kxr) >= cx || fabs(kyr) >= cy ||
                     fabs(kzr) >= cz || (kxr == 0.0 && kyr == 0.0 && kzr == 0.0);
    if (cut)
      for (int c = 0; c < 3; ++c) u[c * nh + m] = mkc<C>(0, 0);
  }
}

// (i k . u) * s for one field (divergence)
template <typename C>
__global__ void k_divhat(const C *u, C *out, long long nh, int nx, int ny, int nz, double ax, double ay,
                         double az, double s) {
  using T = decltype(C{}.x);
  const int nxh = nx / 2 + 1;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < nh;
       m += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(m % nxh), ky = (int)((m / nxh) % ny), kz = (int)(m / ((long long)nxh * ny));
    const double kr[3] = {k_half(kx, nx, ax), k_full(ky, ny, ay), k_full(kz, nz, az)};
    double re = 0, im = 0;
    for (int c = 0; c < 3; ++c) {
      const C v = u[c * nh + m];
      re += -kr[c] * s * (double)v.y;
      im += kr[c] * s * (double)v.x;
    }
    out[m] = mkc<C>(T(re), T(im));
  }
}

// p3dfft STRIDE1 host layout [c][kx][ky][kz] (complex double) <-> internal [c][kz][ky][kx]
template <typename C>
__global__ void k_from_p3dfft(const double2 *src, C *dst, int nxh, int ny, int nz) {
  using T = decltype(C{}.x);
  __shared__ double2 tile[32][33];
  const int c = blockIdx.z / ny, ky = blockIdx.z % ny;
  const int kz0 = blockIdx.x * 32, kx0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int kx = kx0 + i, kz = kz0 + threadIdx.x;
    if (kx < nxh && kz < nz)
      tile[i][threadIdx.x] = src[(((long long)c * nxh + kx) * ny + ky) * nz + kz];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int kz = kz0 + i, kx = kx0 + threadIdx.x;
    if (kx < nxh && kz < nz) {
      const double2 v = tile[threadIdx.x][i];
      dst[(((long long)c * nz + kz) * ny + ky) * nxh + kx] = mkc<C>(T(v.x), T(v.y));
    }
  }
}

template <typename C>
__global__ void k_to_p3dfft(const C *src, double2 *dst, int nxh, int ny, int nz) {
  __shared__ double2 tile[32][33];
  const int c = blockIdx.z / ny, ky = blockIdx.z % ny;
  const int kz0 = blockIdx.x * 32, kx0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int kz = kz0 + i, kx = kx0 + threadIdx.x;
    if (kx < nxh && kz < nz) {
      const C v = src[(((long long)c * nz + kz) * ny + ky) * nxh + kx];
      tile[i][threadIdx.x] = make_double2((double)v.x, (double)v.y);
    }
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int kx = kx0 + i, kz = kz0 + threadIdx.x;
    if (kx < nxh && kz < nz) dst[(((long long)c * nxh + kx) * ny + ky) * nz + kz] = tile[threadIdx.x][i];
  }
}

template <typename A, typename B>
__global__ void k_convert(const A *src, B *dst, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = (B)src[i];
}

// Sets *flag when any component of a state (3 fields nh apart) is nonzero
// (or not a number) at a mode outside the kept set of the pruning rule.
template <typename C>
__global__ void k_cut_check(const C *u, long long nh, long long fstride, int nxh, int ny, AxisKeep kx, AxisKeep ky,
                            AxisKeep kz, int *flag) {
  // m runs over the modes of every box (fstride = nbatch * nh per component)
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < fstride;
       m += (long long)gridDim.x * blockDim.x) {
    const long long mb = m % nh;
    const int ix = (int)(mb % nxh), iy = (int)((mb / nxh) % ny), iz = (int)(mb / ((long long)nxh * ny));
    if (kx.keep(ix) && ky.keep(iy) && kz.keep(iz)) continue;
    for (int c = 0; c < 3; ++c) {
      const C v = u[c * fstride + m];
      if (!(v.x == 0 && v.y == 0)) {
        *flag = 1;
        return;
      }
    }
  }
}

template <typename T> static FinishArgs<T> finish_base(const dnsbox_ctx *c) {
  FinishArgs<T> f;
  memset(&f, 0, sizeof(f));
  const dnsbox_params &p = c->p;
  f.tw = reinterpret_cast<const typename CT<T>::type *>(c->tw[2]);
  f.nh = (long long)c->nh;
  f.nx = p.nx;
  f.ny = p.ny;
  f.nz = p.nz;
  f.nxh = c->nxh;
  f.ax = p.alpha_x;
  f.ay = p.alpha_y;
  f.az = p.alpha_z;
  f.nu = p.nu;
  f.Q = p.Q;
  f.Pin = p.Pin;
  f.kcut = p.kCutOff;
  // rhs.f90:74-88
  f.cutx = (p.nx / 2.0) * (2.0 * p.alpha_x / 3.0);
  f.cuty = (p.ny / 2.0) * (2.0 * p.alpha_y / 3.0);
  f.cutz = (p.nz / 2.0) * (2.0 * p.alpha_z / 3.0);
  f.sph2 = pow((p.nx / 2.0) * 0.5 * p.alpha_x, 2);
  f.bandlim = p.bandlim;
  f.spherical = p.spherical;
  f.ab2_standard = p.ab2_mode == DNSBOX_AB2_STANDARD;
  f.s = 1.0 / ((double)p.nx * p.ny * p.nz);
  f.st = c->st;
  return f;
}

// One right-hand side: passes A-D, E1 (forward z) and E2 (spectral finish).
// cfl: 0 none, 1 record (+control).
template <typename T>
static int run_rhs(dnsbox_ctx *c, const void *uin, int mode, void *out, void *state, void *nold,
                   bool partials, int cfl, dnsbox_diag *drec, bool pruned = false) {
  using C = typename CT<T>::type;
  const dnsbox_params &p = c->p;
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  // rhs_Eband (rhs.f90:22-24) and reset of the CFL maxima
  if (p.bandlim) {
    Prof pr(c, DNSBOX_PASS_SMALL);
    k_eband<C><<<c->nbatch, 256, 0, c->stream>>>(reinterpret_cast<const C *>(uin), (long long)c->fstride, c->band,
                                                 c->nband, p.nx, c->st, s * s, 1, (long long)c->nh);
  } else {
    Prof pr(c, DNSBOX_PASS_SMALL);
    k_reset_umax<<<(c->nbatch + 127) / 128, 128, 0, c->stream>>>(c->st, c->nbatch);
  }
  CK(cudaGetLastError());
  const char *u = reinterpret_cast<const char *>(uin);
  // pass A: inverse z
  StridedArgs<T> a = strided_base<T>(c, 2);
  a.njobs = 5;
  strided_ws<T>(c, a, 2, false, true);   // state -> padded workspace
  set_job<T>(a, 0, cfield(u, c, 0), wfield(c->W1, c, 0));
  set_job<T>(a, 1, cfield(u, c, 1), wfield(c->W1, c, 1));
  set_job<T>(a, 2, cfield(u, c, 2), wfield(c->W1, c, 2));
  set_job<T>(a, 3, cfield(u, c, 1), wfield(c->W1, c, 3), 0.0, -s, 1);   // -dz v
  set_job<T>(a, 4, cfield(u, c, 0), wfield(c->W1, c, 4), 0.0, s, 1);    //  dz u
  if (pruned) {   // input zero outside kept (kz rows, ky, kx); outputs there stay unwritten (zero)
    a.kcol = c->keep[0];
    a.koth = c->keep[1];
    a.krin = c->keep[2];
  }
  RET(run_strided<T>(c, 2, true, a, DNSBOX_PASS_Z_INV, true, uin, 3));
  // pass B: inverse y
  StridedArgs<T> b = strided_base<T>(c, 1);
  strided_ws<T>(c, b, 1, true, true);
  b.njobs = 6;
  set_job<T>(b, 0, wfield(c->W1, c, 0), wfield(c->W2, c, 0));
  set_job<T>(b, 1, wfield(c->W1, c, 1), wfield(c->W2, c, 1));
  set_job<T>(b, 2, wfield(c->W1, c, 2), wfield(c->W2, c, 2));
  // omega_x = dy w - dz v ; omega_y = dz u - dx w ; omega_z = dx v - dy u (ks: 0 kx, 1 ky here)
  set_job<T>(b, 3, wfield(c->W1, c, 2), wfield(c->W2, c, 3), 0.0, s, 1, wfield(c->W1, c, 3));
  set_job<T>(b, 4, wfield(c->W1, c, 4), wfield(c->W2, c, 4), 1.0, 0.0, 0, wfield(c->W1, c, 2), 0.0, -s, 0);
  set_job<T>(b, 5, wfield(c->W1, c, 0), wfield(c->W2, c, 5), 0.0, -s, 1, wfield(c->W1, c, 1), 0.0, s, 0);
  if (pruned) {   // pass-A outputs exist only on kept (ky, kx)
    b.kcol = c->keep[0];
    b.krin = c->keep[1];
  }
  RET(run_strided<T>(c, 1, true, b, DNSBOX_PASS_Y_INV, true, c->W1, 6));
  // pass C: fused x pass
  XlineNLArgs<T> x;
  memset(&x, 0, sizeof(x));
  x.U = reinterpret_cast<const C *>(wfield(c->W2, c, 0));
  x.V = reinterpret_cast<const C *>(wfield(c->W2, c, 1));
  x.W = reinterpret_cast<const C *>(wfield(c->W2, c, 2));
  x.OX = reinterpret_cast<const C *>(wfield(c->W2, c, 3));
  x.OY = reinterpret_cast<const C *>(wfield(c->W2, c, 4));
  x.OZ = reinterpret_cast<const C *>(wfield(c->W2, c, 5));
  x.NX = reinterpret_cast<C *>(wfield(c->W1, c, 0));
  x.NY = reinterpret_cast<C *>(wfield(c->W1, c, 1));
  x.NZ = reinterpret_cast<C *>(wfield(c->W1, c, 2));
  x.pin = x.pout = c->wp;
  x.status = c->tc_status;
  x.tw = reinterpret_cast<const C *>(c->tw[0]);
  x.st = c->st;
  x.lines_per_box = p.ny * p.nz;
  x.nlines = c->nbatch * p.ny * p.nz;
  x.nxh = c->nxh;
  x.alpha_x = p.alpha_x;
  x.s = s;
  if (pruned) x.kxa = c->keep[0].a;   // read only kept kx; write only kx the finish keeps
  {
    Prof pr(c, DNSBOX_PASS_X_NL);
    CK(Ops<T>::xline_nl(p.nx, x, c->sched_x, c->stream));
  }
  if (cfl) {
    const double dx = (2 * M_PI / p.alpha_x) / p.nx, dy = (2 * M_PI / p.alpha_y) / p.ny,
                 dz = (2 * M_PI / p.alpha_z) / p.nz;
    Prof pr(c, DNSBOX_PASS_SMALL);
    k_cfl<<<(c->nbatch + 127) / 128, 128, 0, c->stream>>>(c->st, c->nbatch, dx, dy, dz, !p.tstep_fix,
                                                          c->cfl_first, p.courant_min, p.courant_max, p.dt_max,
                                                          c->ddiag, c->ring_cap);
    CK(cudaGetLastError());
    c->cfl_first = 0;
  }
  // pass D: forward y
  StridedArgs<T> d = strided_base<T>(c, 1);
  strided_ws<T>(c, d, 1, true, true);
  d.njobs = 3;
  for (int f = 0; f < 3; ++f) set_job<T>(d, f, wfield(c->W1, c, f), wfield(c->W2, c, f));
  if (pruned) {   // only kept kx columns; ky rows outside the kept set are masked by the finish
    d.kcol = c->keep[0];
    d.krout = c->keep[1];
  }
  RET(run_strided<T>(c, 1, false, d, DNSBOX_PASS_Y_FWD, true, c->W1, 6));
  // pass E1: forward z of the three components, in place (the SIMT kernel in
  // every form); pruned: kept kx columns and ky tiles, kept kz rows written
  StridedArgs<T> z = strided_base<T>(c, 2);
  strided_ws<T>(c, z, 2, true, true);
  z.njobs = 3;
  for (int f = 0; f < 3; ++f) set_job<T>(z, f, wfield(c->W2, c, f), wfield(c->W2, c, f));
  if (pruned) {
    z.kcol = c->keep[0];
    z.koth = c->keep[1];
    z.krout = c->keep[2];
  }
  RET(run_strided<T>(c, 2, false, z, DNSBOX_PASS_Z_FWD, c->sched_tc[3] != 0, c->W2, 3));
  // pass E2: spectral finish, one warp per (kz, ky) row
  FinishArgs<T> e = finish_base<T>(c);
  e.n3 = reinterpret_cast<const C *>(c->W2);
  e.n3_pitch = c->wp;
  e.n3_nh = (long long)c->wstride;
  e.n3_bstride = (long long)p.nz * p.ny * c->wp;
  e.uin = reinterpret_cast<const C *>(uin);
  e.out = reinterpret_cast<C *>(out);
  e.state = reinterpret_cast<C *>(state);
  e.nold = reinterpret_cast<C *>(nold);
  e.force = reinterpret_cast<const C *>(c->force);
  e.partials = partials ? c->partials : nullptr;
  e.nu_box = c->d_nu;
  e.nh = (long long)c->fstride;
  e.bstride = (long long)c->nh;
  e.mode = mode;
  e.kx = pruned ? c->keep[0] : AxisKeep{0, p.nx, 0};
  e.ky = pruned ? c->keep[1] : AxisKeep{0, p.ny, 1};
  e.kz = pruned ? c->keep[2] : AxisKeep{0, p.nz, 1};
  const int nrows = e.kz.count() * e.ky.count();
  Prof pr(c, DNSBOX_PASS_Z_FIN);
  const dim3 grid((unsigned)((nrows + 7) / 8), (unsigned)c->nbatch);
  switch (mode) {
    case FIN_RHS: k_finish_rows<T, FIN_RHS><<<grid, 256, 0, c->stream>>>(e, nrows); break;
    case FIN_PRED: k_finish_rows<T, FIN_PRED><<<grid, 256, 0, c->stream>>>(e, nrows); break;
    case FIN_CORR: k_finish_rows<T, FIN_CORR><<<grid, 256, 0, c->stream>>>(e, nrows); break;
    default: k_finish_rows<T, FIN_AB2><<<grid, 256, 0, c->stream>>>(e, nrows); break;
  }
  CK(cudaGetLastError());
  return DNSBOX_OK;
}

// ------------------------------------------------------------ TMA passes
// cuTensorMapEncodeTiled, from the driver through the runtime (no link
// dependency on libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// First rows of the 8-row boxes that cover the rows a pass keeps on a full
// axis of length n (all rows when k.a = 0): [0, a), the Nyquist row n/2 and
// (n - a, n), each range rounded out to whole boxes.  Returns the count, or
// the full cover when the rounded ranges would overlap.
static int tma_row_boxes(const AxisKeep &k, int n, int br, unsigned short *rows) {
  int nb = 0;
  if (k.a > 0) {
    const int lo_end = (k.a + br - 1) / br * br;
    int hi_start = n;
    while (hi_start - br >= 0 && hi_start > n - k.a + 1) hi_start -= br;
    const int nq = n / 2;
    if (lo_end <= nq && nq + br <= hi_start && nq % br == 0) {
      for (int r = 0; r < lo_end; r += br) rows[nb++] = (unsigned short)r;
      rows[nb++] = (unsigned short)nq;
      for (int r = hi_start; r < n; r += br) rows[nb++] = (unsigned short)r;
      return nb;
    }
  }
  for (int r = 0; r < n; r += br) rows[nb++] = (unsigned short)r;
  return nb;
}

int run_strided_tma(dnsbox_ctx *c, int axis, bool inv, const StridedArgs<float> &a, const void *base, int nslots,
                    int kind) {
  // a z pass reads the state (pitch nxh, components fstride apart) unless its
  // inputs live in the padded workspace (W2: the forward z pass)
  const bool ws_z = axis == 2 && base != nullptr && (base == c->W1 || base == c->W2);
  const dnsbox_params &p = c->p;
  const int n = axis == 2 ? p.nz : p.ny;
  const int width = 4096 / n;   // TmaPlan<n>::TCW
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return set_err(DNSBOX_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  TmaArgs t;
  memset(&t, 0, sizeof(t));
  // tile grid (as run_strided)
  t.kcol = a.kcol;
  t.koth = a.koth;
  t.krin = a.krin;
  t.krout = a.krout;
  if (a.kcol.a) {
    t.ntx_lo = (a.kcol.a + width - 1) / width;
    const int nt = (p.nx / 2) / width;
    t.nyq_tile = nt < t.ntx_lo ? 0 : (a.kcol.a % width ? -1 : nt);
  }
  const int ntx = t.ntx_lo ? t.ntx_lo + (t.nyq_tile > 0 ? 1 : 0) : (c->nxh + width - 1) / width;
  const int nother = a.koth.a ? a.koth.count() : (axis == 2 ? p.ny : p.nz);
  const int nbatch = a.nbatch > 0 ? a.nbatch : 1;
  const long long total = (long long)a.njobs * ntx * nother * nbatch;
  if (total >= (1LL << 31)) return set_err(DNSBOX_ERR_SIZE, "TMA pass: too many tiles");
  t.total = (int)total;
  t.per_box.init((unsigned)(a.njobs * ntx * nother));
  t.njobs_d.init((unsigned)a.njobs);
  t.ntxd.init((unsigned)ntx);
  // jobs: slot coordinates of the inputs within `base`
  const size_t slot_bytes = (axis == 2 && !ws_z ? c->fstride : c->wstride) * sizeof(float2);
  auto slot_of = [&](const void *ptr) -> int {
    const long long d = reinterpret_cast<const char *>(ptr) - reinterpret_cast<const char *>(base);
    if (d < 0 || d % (long long)slot_bytes || d / (long long)slot_bytes >= nslots) return -2;
    return (int)(d / (long long)slot_bytes);
  };
  t.njobs = a.njobs;
  for (int j = 0; j < a.njobs; ++j) {
    const StridedJob<float> &J = a.job[j];
    TmaJob &T = t.job[j];
    T.in1 = J.in1;
    T.in2 = J.in2;
    T.out = J.out;
    T.a1 = (float)J.a1;
    T.b1 = (float)J.b1;
    T.a2 = (float)J.a2;
    T.b2 = (float)J.b2;
    T.ks1 = J.ks1;
    T.ks2 = J.ks2;
    T.slot1 = slot_of(J.in1);
    T.slot2 = J.in2 ? slot_of(J.in2) : -1;
    if (T.slot1 < 0 || T.slot2 < -1) return set_err(DNSBOX_ERR_STATE, "TMA pass: job input outside its tensor");
    if (J.in2) t.two = 1;
  }
  t.tw = reinterpret_cast<const float2 *>(a.tw);
  t.rowstride = a.rowstride;
  t.otherstride = a.otherstride;
  t.bstride = a.bstride;
  t.rso = out_rowstride(a);
  t.oso = out_otherstride(a);
  t.bso = out_bstride(a);
  if ((t.rso | t.oso | t.bso) & 1) return set_err(DNSBOX_ERR_STATE, "TMA pass: output rows must be 16-byte aligned");
  if ((long long)n * t.rso >= (1LL << 31)) return set_err(DNSBOX_ERR_SIZE, "TMA pass: 32-bit row offsets");
  t.plane = axis == 2;
  t.in_pitch = ws_z ? c->wp : c->nxh;
  t.ncols = a.ncols;
  t.nx = a.nx;
  t.n_other = a.n_other;
  t.alpha_row = (float)a.alpha_row;
  t.alpha_x = (float)a.alpha_x;
  t.alpha_other = (float)a.alpha_other;
  t.box_rows = c->tma_box_rows;
  t.nbox = tma_row_boxes(a.krin, n, t.box_rows, t.box_row);
  // the input tensor map
  const int spc = width + 2;
  cuuint64_t dims[5], strides[4];
  const cuuint32_t box[5] = {(cuuint32_t)(2 * spc), (cuuint32_t)t.box_rows, 1, 1, 1}, estr[5] = {1, 1, 1, 1, 1};
  if (axis == 2) {   // (plane floats, z, box, slot, 1): the state, or the padded workspace
    const unsigned long long pitch = ws_z ? c->wp : c->nxh;
    const unsigned long long plane = (unsigned long long)p.ny * pitch;
    const unsigned long long boxs = plane * p.nz, slots = ws_z ? c->wstride : c->fstride;
    dims[0] = 2 * plane;
    dims[1] = (cuuint64_t)p.nz;
    dims[2] = (cuuint64_t)nbatch;
    dims[3] = (cuuint64_t)nslots;
    dims[4] = 1;
    strides[0] = plane * 8;
    strides[1] = boxs * 8;
    strides[2] = slots * 8;
    strides[3] = slots * 8 * nslots;
  } else {           // padded workspace: (row floats, y, z, box, slot)
    dims[0] = 2ull * c->nxh;
    dims[1] = (cuuint64_t)p.ny;
    dims[2] = (cuuint64_t)p.nz;
    dims[3] = (cuuint64_t)nbatch;
    dims[4] = (cuuint64_t)nslots;
    strides[0] = (cuuint64_t)c->wp * 8;
    strides[1] = (cuuint64_t)p.ny * c->wp * 8;
    strides[2] = (cuuint64_t)p.nz * p.ny * c->wp * 8;
    strides[3] = (cuuint64_t)c->wstride * 8;
  }
  const CUresult r = encode(&t.map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, const_cast<void *>(base), dims, strides, box,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_err(DNSBOX_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  Prof pr(c, kind);
  CK(Ops<float>::strided_tma(n, t, inv, c->adft, c->tc_status, c->tma_ctas_per_sm * c->nsm, c->stream));
  return DNSBOX_OK;
}

// Synchronises the stream and reports a tensor-core pass whose MMA
// completion wait gave up (the flag is cleared).  Every entry point that
// synchronises before returning ends with it; asynchronous entries leave the
// flag to the next such call or to dnsbox_sync.
int tc_check(dnsbox_ctx *c) {
  int *flag = reinterpret_cast<int *>(c->hstage + 63);
  *flag = 0;
  if (c->tc_status) CK(cudaMemcpyAsync(flag, c->tc_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (*flag) {
    CK(cudaMemsetAsync(c->tc_status, 0, sizeof(int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const int code = *flag;
    return set_err(DNSBOX_ERR_TIMEOUT, "a bounded device wait gave up (%s)",
                   code == 2 ? "staged TMA copy" : code == 3 ? "tensor-core MMA of a TMA pass" : "tensor-core MMA");
  }
  return DNSBOX_OK;
}

// Copies the records of steps [first, first + n) (n <= ring_cap) from the
// device ring into host[(step - first) * nbatch + box].
static int ring_read(dnsbox_ctx *c, long long first, int n, dnsbox_diag *host) {
  int done = 0;
  while (done < n) {
    const long long step = first + done;
    const int pos = (int)(step % c->ring_cap);
    int run = c->ring_cap - pos;
    if (run > n - done) run = n - done;
    CK(cudaMemcpyAsync(host + (size_t)done * c->nbatch, c->ddiag + (size_t)pos * c->nbatch,
                       (size_t)run * c->nbatch * sizeof(dnsbox_diag), cudaMemcpyDeviceToHost, c->stream));
    done += run;
  }
  RET(tc_check(c));
  return DNSBOX_OK;
}

// The semi-implicit step (dnsboximplicit.f90:88-181) of one box: N(u_n), the
// first guess, fixed-point iterations until the summed component change is at
// most implicit_tol (one host read-back per iteration, at most
// implicit_max_iter), state_project; then the row sums the step record needs.
template <typename T> static int semi_implicit_step(dnsbox_ctx *c, void *uh) {
  using C = typename CT<T>::type;
  const dnsbox_params &p = c->p;
  const long long nh = (long long)c->nh;
  C *u = reinterpret_cast<C *>(c->ustar);
  const C *un = reinterpret_cast<const C *>(uh), *n0 = reinterpret_cast<const C *>(c->nold);
  const C *nk = reinterpret_cast<const C *>(c->sibuf);
  RET(ensure_red(c, 3));
  double *chg = c->red;   // 3 doubles
  double *hchg = c->hstage + 48;
  RET(run_rhs<T>(c, uh, FIN_RHS, c->nold, nullptr, nullptr, false, 1, nullptr, c->prune_now));   // :93
  {
    Prof pr(c, DNSBOX_PASS_SMALL);
    k_si_update<C, true><<<grid_for(nh), 256, 0, c->stream>>>(u, un, n0, nullptr, nh, p.nx, p.ny, p.nz, p.alpha_x,
                                                             p.alpha_y, p.alpha_z, p.nu, p.Q, p.implicit_c, c->st,
                                                             nullptr);
    CK(cudaGetLastError());
  }
  int it = 0;
  while (it < p.implicit_max_iter) {   // :126-175
    ++it;
    RET(run_rhs<T>(c, u, FIN_RHS, c->sibuf, nullptr, nullptr, false, 0, nullptr, c->prune_now));
    CK(cudaMemsetAsync(chg, 0, 3 * sizeof(double), c->stream));
    {
      Prof pr(c, DNSBOX_PASS_SMALL);
      k_si_update<C, false><<<grid_for(nh), 256, 0, c->stream>>>(u, un, n0, nk, nh, p.nx, p.ny, p.nz, p.alpha_x,
                                                                p.alpha_y, p.alpha_z, p.nu, p.Q, p.implicit_c,
                                                                c->st, chg);
      CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(hchg, chg, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const double total = hchg[0] + hchg[1] + hchg[2];
    if (!(total == total)) return set_err(DNSBOX_ERR_NONFINITE, "semi-implicit iteration: non-finite change");
    if (total <= p.implicit_tol) break;
  }
  c->si_iters = it;
  Prof pr(c, DNSBOX_PASS_SMALL, 2);
  k_project<C><<<grid_for(nh), 256, 0, c->stream>>>(u, nh, p.nx, p.ny, p.nz, p.alpha_x, p.alpha_y, p.alpha_z);   // :177
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(uh, u, 3 * (size_t)nh * sizeof(C), cudaMemcpyDeviceToDevice, c->stream));
  if (!c->proj_every) {   // otherwise step_once sums the rows after the projection
    k_row_sums<C><<<(p.ny * p.nz + 7) / 8, 256, 0, c->stream>>>(reinterpret_cast<const C *>(uh), nh, nh, p.nx, p.ny,
                                                                p.nz, p.alpha_x, p.alpha_y, p.alpha_z, c->partials);
    CK(cudaGetLastError());
  }
  return DNSBOX_OK;
}

// One step of every box of the context (no host synchronisation, except the
// semi-implicit step's per-iteration read-back).
template <typename T> static int step_once(dnsbox_ctx *c, void *uh) {
  const dnsbox_params &p = c->p;
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  const bool pc = (p.stepper == DNSBOX_HEUN) || (p.stepper == DNSBOX_AB2 && !c->ab2_started);
  if (p.stepper == DNSBOX_SEMI_IMPLICIT) {
    RET(semi_implicit_step<T>(c, uh));
  } else if (pc) {
    // dnsboxheun.f90:85-126 (and dnsbox.f90:87-141 for the AB2 first step)
    RET(run_rhs<T>(c, uh, FIN_PRED, c->ustar, nullptr, p.stepper == DNSBOX_AB2 ? c->nold : nullptr, false, 1,
                   nullptr, c->prune_now));
    RET(run_rhs<T>(c, c->ustar, FIN_CORR, nullptr, uh, nullptr, true, 0, nullptr, c->prune_now));
    if (p.stepper == DNSBOX_AB2) c->ab2_started = 1;
  } else {
    // dnsbox.f90:143-191
    RET(run_rhs<T>(c, uh, FIN_AB2, nullptr, uh, c->nold, true, 1, nullptr, c->prune_now));
  }
  if (c->proj_every) {
    // dnsboxband.f90:142-143: project and dealias the new state, then its row sums
    using C = typename CT<T>::type;
    const dim3 g((unsigned)grid_for((long long)c->nh, 256, 148 * 8), (unsigned)c->nbatch);
    Prof pr(c, DNSBOX_PASS_SMALL, 2);
    k_project_dealias<C><<<g, 256, 0, c->stream>>>(reinterpret_cast<C *>(uh), (long long)c->nh,
                                                    (long long)c->fstride, p.nx, p.ny, p.nz, p.alpha_x, p.alpha_y,
                                                    p.alpha_z, p.spherical, (p.nx / 2.0) * (2.0 * p.alpha_x / 3.0),
                                                    (p.ny / 2.0) * (2.0 * p.alpha_y / 3.0),
                                                    (p.nz / 2.0) * (2.0 * p.alpha_z / 3.0),
                                                    pow((p.nx / 2.0) * (2.0 / 3.0) * p.alpha_x, 2));
    CK(cudaGetLastError());
    k_row_sums<C><<<dim3((unsigned)((p.ny * p.nz + 7) / 8), (unsigned)c->nbatch), 256, 0, c->stream>>>(
        reinterpret_cast<const C *>(uh), (long long)c->nh, (long long)c->fstride, p.nx, p.ny, p.nz, p.alpha_x,
        p.alpha_y, p.alpha_z, c->partials);
    CK(cudaGetLastError());
  }
  // k_row_sums visits every row
  const bool rows_pruned = c->prune_now && p.stepper != DNSBOX_SEMI_IMPLICIT && !c->proj_every;
  const AxisKeep ky = rows_pruned ? c->keep[1] : AxisKeep{0, p.ny, 1};
  const AxisKeep kz = rows_pruned ? c->keep[2] : AxisKeep{0, p.nz, 1};
  double *planes = c->partials + 2 * (size_t)c->npartials * c->nbatch;
  Prof pr(c, DNSBOX_PASS_SMALL, 2);
  k_plane_sums<<<dim3((unsigned)p.nz, (unsigned)c->nbatch), 256, 0, c->stream>>>(c->partials, planes, p.nz, p.ny, ky,
                                                                                 kz);
  CK(cudaGetLastError());
  k_finalize<<<c->nbatch, 1024, 0, c->stream>>>(c->st, planes, p.nz, s * s, p.nu, c->d_nu, p.Q, p.Pin, p.bandlim,
                                                 c->ddiag, c->ring_cap);
  CK(cudaGetLastError());
  c->host_step += 1;
  return DNSBOX_OK;
}

// Decides whether this call may use the pruned passes: the state must vanish
// exactly on the 2/3-rule cut set (the stepper then keeps it so).
// The check of every box of the context writes c->cut_flag (nonzero: some
// box has content on the cut set); queued on c->stream.
template <typename T> static int cut_check_async(dnsbox_ctx *c, const void *uh) {
  using C = typename CT<T>::type;
  CK(cudaMemsetAsync(c->cut_flag, 0, sizeof(int), c->stream));
  k_cut_check<C><<<grid_for((long long)c->fstride), 256, 0, c->stream>>>(
      reinterpret_cast<const C *>(uh), (long long)c->nh, (long long)c->fstride, c->nxh, c->p.ny, c->keep[0],
      c->keep[1], c->keep[2], c->cut_flag);
  CK(cudaGetLastError());
  return DNSBOX_OK;
}

template <typename T> static int prune_decide(dnsbox_ctx *c, const void *uh) {
  c->prune_now = 0;
  if (!c->prune_ok || c->p.no_prune) return DNSBOX_OK;
  RET(cut_check_async<T>(c, uh));
  int *flag = reinterpret_cast<int *>(c->hstage + 62);
  CK(cudaMemcpyAsync(flag, c->cut_flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->prune_now = *flag == 0;
  return DNSBOX_OK;
}

template <typename T> static int step_impl(dnsbox_ctx *c, void *uh, int nsteps, dnsbox_diag *dh) {
  RET(prune_decide<T>(c, uh));
  long long chunk_first = c->host_step;
  for (int n = 0; n < nsteps; ++n) {
    RET(step_once<T>(c, uh));
    const int in_chunk = (int)(c->host_step - chunk_first);
    if (dh && (in_chunk == c->ring_cap || n == nsteps - 1)) {
      RET(ring_read(c, chunk_first, in_chunk, dh + (size_t)(n + 1 - in_chunk) * c->nbatch));
      chunk_first = c->host_step;
    }
  }
  if (dh) {
    for (int n = 0; n < nsteps * c->nbatch; ++n)
      if (dh[n].nonfinite) return set_err(DNSBOX_ERR_NONFINITE, "non-finite energy at step %d", dh[n].step);
  }
  return DNSBOX_OK;
}

// --------------------------------------------------------------- create
static int alloc_twiddles(dnsbox_ctx *c, int axis, int n) {
  std::vector<double> h(2 * (size_t)n);
  for (int j = 0; j < n; ++j) {
    const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)j / (long double)n;
    h[2 * j] = (double)cosl(a);
    h[2 * j + 1] = (double)sinl(a);
  }
  CK(cudaMalloc(&c->tw[axis], (size_t)n * c->cbytes));
  if (c->fp64) {
    CK(cudaMemcpy(c->tw[axis], h.data(), (size_t)n * 16, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> f(2 * (size_t)n);
    for (size_t i = 0; i < f.size(); ++i) f[i] = (float)h[i];
    CK(cudaMemcpy(c->tw[axis], f.data(), (size_t)n * 8, cudaMemcpyHostToDevice));
  }
  return DNSBOX_OK;
}

// DFT-64 operands of the tensor-core passes (kernels_tc.cuh): for each
// direction the real and imaginary parts of F[k][n] = exp(-+2 pi i k n / 64)
// as rows 2k and 2k + 1 of A, split into f16 hi = rn(A) and lo = rn(A - hi),
// each stored as a 128 x 64 K-major operand.
static int alloc_dft64(dnsbox_ctx *c) {
  std::vector<__half> h((size_t)kTcDftBytes / 2);
  for (int dir = 0; dir < 2; ++dir) {
    __half *hi = h.data() + (size_t)dir * 2 * 128 * 64;
    __half *lo = hi + 128 * 64;
    const double sgn = dir == 0 ? -1.0 : 1.0;
    for (int k = 0; k < 64; ++k)
      for (int n = 0; n < 64; ++n) {
        const long double ang = 2.0L * 3.141592653589793238462643383279502884L * (long double)((k * n) % 64) / 64.0L;
        const double val[2] = {(double)cosl(ang), sgn * (double)sinl(ang)};
        for (int rb = 0; rb < 2; ++rb) {
          const __half vh = __double2half(val[rb]);
          const __half vl = __double2half(val[rb] - (double)__half2float(vh));
          const int off = tc::kmajor_offset(2 * k + rb, n, 128) / 2;
          hi[off] = vh;
          lo[off] = vl;
        }
      }
  }
  CK(cudaMalloc(&c->adft, (size_t)kTcDftBytes));
  CK(cudaMemcpy(c->adft, h.data(), (size_t)kTcDftBytes, cudaMemcpyHostToDevice));
  CK(cudaMalloc(&c->tc_status, sizeof(int)));
  CK(cudaMemset(c->tc_status, 0, sizeof(int)));
  int dev = 0, nsm = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  c->tc_ctas = TcPlan<256>::CTAS_PER_SM * nsm;   // persistent: every resident CTA slot
  c->nsm = nsm;
  // DNSBOX_TC_KERNEL=legacy keeps the right-hand side on the cp.async-fed
  // tensor-core kernel of the standalone transforms (for comparisons)
  const char *kern = getenv("DNSBOX_TC_KERNEL");
  c->tma_on = !(kern && strcmp(kern, "legacy") == 0);
  // rows per TMA box of the staged tiles (8, 16, 32 or 64; DNSBOX_TMA_BOX_ROWS)
  const char *br = getenv("DNSBOX_TMA_BOX_ROWS");
  const int brv = br ? atoi(br) : 32;
  c->tma_box_rows = (brv == 8 || brv == 16 || brv == 32 || brv == 64) ? brv : 32;
  // resident CTAs per SM of the TMA passes (DNSBOX_TMA_CTAS_PER_SM = 2 for
  // two; one by default: with two per SM, repeated 256^3 pruned steps gave an
  // occasional wrong result that one CTA per SM never showed)
  const char *cps = getenv("DNSBOX_TMA_CTAS_PER_SM");
  c->tma_ctas_per_sm = (cps && atoi(cps) == 2) ? 2 : 1;
  return DNSBOX_OK;
}

static void free_ctx(dnsbox_ctx *c) {
  if (!c) return;
  cudaFree(c->adft);
  cudaFree(c->tc_status);
  cudaFree(c->cut_flag);
  for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
  cudaFree(c->W1);
  cudaFree(c->W2);
  cudaFree(c->ustar);
  cudaFree(c->nold);
  cudaFree(c->sibuf);
  for (int i = 0; i < 3; ++i) cudaFree(c->tw[i]);
  cudaFree(c->st);
  cudaFree(c->partials);
  cudaFree(c->red);
  cudaFree(c->band);
  cudaFree(c->ddiag);
  descent_graphs_free(c);
  cudaFree(c->adj);
  cudaFree(c->orbit);
  cudaFree(c->d_nu);
  if (c->hstage) cudaFreeHost(c->hstage);
  delete c;
}

extern "C" int dnsbox_create(const dnsbox_params *p, dnsbox_ctx **out) {
  if (!p || !out) return set_err(DNSBOX_ERR_ARG, "null argument");
  *out = nullptr;
  if (!dnsbox_supported_size(p->nx) || !dnsbox_supported_size(p->ny) || !dnsbox_supported_size(p->nz))
    return set_err(DNSBOX_ERR_SIZE, "unsupported grid %dx%dx%d", p->nx, p->ny, p->nz);
  if (p->precision != DNSBOX_FP64 && p->precision != DNSBOX_FP32 && p->precision != DNSBOX_TC_SPLIT)
    return set_err(DNSBOX_ERR_UNSUPPORTED, "precision %d not available", p->precision);
  if (!(p->nu >= 0.0) || !(p->Deltak > 0.0) || !(p->dt > 0.0) || !(p->alpha_x > 0) || !(p->alpha_y > 0) ||
      !(p->alpha_z > 0))
    return set_err(DNSBOX_ERR_ARG, "invalid physical parameter");
  if (p->stepper != DNSBOX_HEUN && p->stepper != DNSBOX_AB2 && p->stepper != DNSBOX_SEMI_IMPLICIT)
    return set_err(DNSBOX_ERR_ARG, "invalid stepper %d", p->stepper);
  if (p->stepper == DNSBOX_SEMI_IMPLICIT &&
      (p->nbatch > 1 || p->implicit_max_iter < 1 || !(p->implicit_tol >= 0.0) || !(p->implicit_c > 0.0) ||
       !(p->implicit_c <= 1.0)))
    return set_err(DNSBOX_ERR_ARG, "semi-implicit stepper: one box, implicit_max_iter >= 1, implicit_tol >= 0, "
                                   "0 < implicit_c <= 1");
  CK(cudaSetDevice(p->device));
  if (p->nbatch < 0 || p->nbatch > 65535) return set_err(DNSBOX_ERR_ARG, "nbatch %d out of range", p->nbatch);
  dnsbox_ctx *c = new dnsbox_ctx();
  c->p = *p;
  c->nbatch = p->nbatch > 1 ? p->nbatch : 1;
  c->fp64 = p->precision == DNSBOX_FP64;
  c->cbytes = c->fp64 ? 16 : 8;
  c->nxh = p->nx / 2 + 1;
  c->nh = (size_t)p->nz * p->ny * c->nxh;
  c->np = (size_t)p->nz * p->ny * p->nx;
  c->fstride = c->nh * c->nbatch;
  {
    const int q = c->fp64 ? 8 : 16;   // complex elements per 128 bytes
    c->wp = (c->nxh + q - 1) / q * q;
    c->wstride = (size_t)c->nbatch * p->nz * p->ny * c->wp;
  }
  int rc = DNSBOX_OK;
  auto fail = [&](int r) {
    free_ctx(c);
    return r;
  };
  const size_t fb = c->fstride * c->cbytes;
  const size_t wb = (c->wstride > c->fstride ? c->wstride : c->fstride) * c->cbytes;   // one workspace slot
  c->ring_cap = 1024;
  cudaError_t e;
  if ((e = cudaMalloc(&c->W1, 6 * wb)) != cudaSuccess ||
      (e = cudaMalloc(&c->W2, 6 * wb)) != cudaSuccess ||
      (e = cudaMalloc(&c->ustar, 3 * fb)) != cudaSuccess ||
      (p->stepper != DNSBOX_HEUN && (e = cudaMalloc(&c->nold, 3 * fb)) != cudaSuccess) ||
      (p->stepper == DNSBOX_SEMI_IMPLICIT && (e = cudaMalloc(&c->sibuf, 3 * fb)) != cudaSuccess) ||
      (e = cudaMalloc(&c->st, c->nbatch * sizeof(StepState))) != cudaSuccess ||
      (e = cudaMalloc(&c->ddiag, (size_t)c->ring_cap * c->nbatch * sizeof(dnsbox_diag))) != cudaSuccess ||
      (c->nbatch > 1 && (e = cudaMalloc(&c->d_nu, c->nbatch * sizeof(double))) != cudaSuccess)) {
    cudaGetLastError();
    return fail(set_err(DNSBOX_ERR_OOM, "device allocation failed: %s", cudaGetErrorString(e)));
  }
  if ((rc = alloc_twiddles(c, 0, p->nx)) || (rc = alloc_twiddles(c, 1, p->ny)) ||
      (rc = alloc_twiddles(c, 2, p->nz)))
    return fail(rc);
  if (p->precision == DNSBOX_TC_SPLIT) {
    c->tc = 1;
    if ((rc = alloc_dft64(c))) return fail(rc);
  } else {   // the status flag of bounded device waits (the staged x pass)
    if ((e = cudaMalloc(&c->tc_status, sizeof(int))) != cudaSuccess || (e = cudaMemset(c->tc_status, 0, sizeof(int))) != cudaSuccess)
      return fail(set_err(DNSBOX_ERR_OOM, "device allocation failed: %s", cudaGetErrorString(e)));
  }
  // pruning rule per axis, derived from the dealiasing mask and checked against it
  {
    const int ns[3] = {p->nx, p->ny, p->nz};
    const double al[3] = {p->alpha_x, p->alpha_y, p->alpha_z};
    bool ok = true;
    for (int ax = 0; ax < 3; ++ax) {
      const int n = ns[ax];
      const bool full = ax > 0;
      const double cut = (n / 2.0) * (2.0 * al[ax] / 3.0);
      auto kk = [&](int i) { return full ? k_full(i, n, al[ax]) : k_half(i, n, al[ax]); };
      int a = 0;
      for (int i = 1; i < n / 2; ++i)
        if (fabs(kk(i)) >= cut) {
          a = i;
          break;
        }
      c->keep[ax] = AxisKeep{a, n, full ? 1 : 0};
      const int m = full ? n : n / 2 + 1;
      for (int i = 0; i < m; ++i)
        if (c->keep[ax].keep(i) != !(fabs(kk(i)) >= cut)) ok = false;
      if (a == 0) ok = false;
    }
    c->prune_ok = ok;
    if (!ok)
      for (int ax = 0; ax < 3; ++ax) c->keep[ax].a = 0;
    if ((e = cudaMalloc(&c->cut_flag, sizeof(int))) != cudaSuccess)
      return fail(set_err(DNSBOX_ERR_OOM, "device allocation failed"));
    // pruned steps leave the cut set of these buffers untouched: start at zero
    if ((e = cudaMemset(c->ustar, 0, 3 * fb)) != cudaSuccess ||
        (c->nold && (e = cudaMemset(c->nold, 0, 3 * fb)) != cudaSuccess) ||
        (c->sibuf && (e = cudaMemset(c->sibuf, 0, 3 * fb)) != cudaSuccess))
      return fail(set_err(DNSBOX_ERR_CUDA, "%s", cudaGetErrorString(e)));
  }
  c->npartials = p->nz * p->ny;   // one (E, D) pair per (kz, ky) row, then one per kz plane
  if ((e = cudaMalloc(&c->partials, 2 * (size_t)(c->npartials + p->nz) * c->nbatch * sizeof(double))) != cudaSuccess)
    return fail(set_err(DNSBOX_ERR_OOM, "device allocation failed"));
  // band modes |k| <= kCutOff (rhs.f90:145-149), stored as (offset lo, offset hi, kx)
  std::vector<int> band;
  auto cand = [](int n, double a, double kc, bool half) {
    std::vector<int> v;
    const int m = half ? n / 2 + 1 : n;
    for (int i = 0; i < m; ++i) {
      const double k = half ? k_half(i, n, a) : k_full(i, n, a);
      if (fabs(k) <= kc) v.push_back(i);
    }
    return v;
  };
  if (p->bandlim) {
    for (int kz : cand(p->nz, p->alpha_z, p->kCutOff, false))
      for (int ky : cand(p->ny, p->alpha_y, p->kCutOff, false))
        for (int kx : cand(p->nx, p->alpha_x, p->kCutOff, true)) {
          const double a = k_half(kx, p->nx, p->alpha_x), b = k_full(ky, p->ny, p->alpha_y),
                       cc = k_full(kz, p->nz, p->alpha_z);
          if (sqrt(a * a + b * b + cc * cc) > p->kCutOff) continue;
          const long long off = ((long long)kz * p->ny + ky) * c->nxh + kx;
          band.push_back((int)(off & 0xffffffffLL));
          band.push_back((int)(off >> 32));
          band.push_back(kx);
        }
    c->nband = (int)band.size() / 3;
    if (c->nband) {
      if ((e = cudaMalloc(&c->band, band.size() * sizeof(int))) != cudaSuccess)
        return fail(set_err(DNSBOX_ERR_OOM, "device allocation failed"));
      if ((e = cudaMemcpy(c->band, band.data(), band.size() * sizeof(int), cudaMemcpyHostToDevice)) !=
          cudaSuccess)
        return fail(set_err(DNSBOX_ERR_CUDA, "%s", cudaGetErrorString(e)));
    }
  }
  {
    std::vector<StepState> hs(c->nbatch);
    memset(hs.data(), 0, hs.size() * sizeof(StepState));
    for (auto &x : hs) x.dt = p->dt;
    if ((e = cudaMemcpy(c->st, hs.data(), hs.size() * sizeof(StepState), cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail(set_err(DNSBOX_ERR_CUDA, "%s", cudaGetErrorString(e)));
    if (c->d_nu) {
      std::vector<double> nus(c->nbatch, p->nu);
      if ((e = cudaMemcpy(c->d_nu, nus.data(), nus.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(set_err(DNSBOX_ERR_CUDA, "%s", cudaGetErrorString(e)));
    }
  }
  if ((e = cudaMallocHost(&c->hstage, 64 * sizeof(double))) != cudaSuccess)
    return fail(set_err(DNSBOX_ERR_CUDA, "%s", cudaGetErrorString(e)));
  // variables.f90:112-123
  if (p->spherical)
    c->nspec = (int)(((p->nx / 2.0) * (2.0 * p->alpha_x / 3.0)) / p->Deltak) - 1;
  else
    c->nspec = (int)(sqrt(pow((p->nx / 2.0) * (2.0 * p->alpha_x / 3.0), 2) +
                          pow((p->ny / 2.0) * (2.0 * p->alpha_y / 3.0), 2) +
                          pow((p->nz / 2.0) * (2.0 * p->alpha_z / 3.0), 2)) /
                     p->Deltak) -
               1;
  schedule_from_cache(c);   // a schedule tuned earlier for this device and shape
  *out = c;
  return DNSBOX_OK;
}

extern "C" int dnsbox_destroy(dnsbox_ctx *ctx) {
  if (!ctx) return DNSBOX_OK;
  cudaSetDevice(ctx->p.device);
  cudaStreamSynchronize(ctx->stream);
  free_ctx(ctx);
  return DNSBOX_OK;
}

extern "C" int dnsbox_set_stream(dnsbox_ctx *ctx, void *stream) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  ctx->stream = reinterpret_cast<cudaStream_t>(stream);
  return DNSBOX_OK;
}

extern "C" int dnsbox_field_bytes(const dnsbox_ctx *ctx, size_t *sb, size_t *pb) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  if (sb) *sb = ctx->nh * ctx->cbytes;
  if (pb) *pb = ctx->np * ctx->cbytes / 2;
  return DNSBOX_OK;
}

extern "C" int dnsbox_nspec(const dnsbox_ctx *ctx) { return ctx ? ctx->nspec : -1; }

extern "C" int dnsbox_step_pruned(const dnsbox_ctx *ctx) { return ctx ? ctx->prune_now : -1; }
extern "C" int dnsbox_implicit_iterations(const dnsbox_ctx *ctx) { return ctx ? ctx->si_iters : -1; }

#define BEGIN(ctx)                                              \
  if (!(ctx)) return set_err(DNSBOX_ERR_ARG, "null context");   \
  CK(cudaSetDevice((ctx)->p.device));
// entry points that take one box's fields
#define SINGLE(ctx)                                                                              \
  if ((ctx)->nbatch > 1)                                                                         \
    return set_err(DNSBOX_ERR_UNSUPPORTED, "not available on a batched context (nbatch = %d)", \
                   (ctx)->nbatch);

extern "C" int dnsbox_set_dt(dnsbox_ctx *ctx, double dt) {
  BEGIN(ctx);
  if (!(dt > 0.0) || !isfinite(dt)) return set_err(DNSBOX_ERR_ARG, "dt must be positive and finite");
  k_set_state<<<(ctx->nbatch + 127) / 128, 128, 0, ctx->stream>>>(ctx->st, ctx->nbatch, offsetof(StepState, dt), dt);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return DNSBOX_OK;
}

extern "C" int dnsbox_get_dt(dnsbox_ctx *ctx, double *dt) {
  BEGIN(ctx);
  if (!dt) return set_err(DNSBOX_ERR_ARG, "null output");
  CK(cudaMemcpyAsync(ctx->hstage, &ctx->st->dt, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *dt = ctx->hstage[0];
  return DNSBOX_OK;
}

extern "C" int dnsbox_set_time(dnsbox_ctx *ctx, double t) {
  BEGIN(ctx);
  k_set_state<<<(ctx->nbatch + 127) / 128, 128, 0, ctx->stream>>>(ctx->st, ctx->nbatch, offsetof(StepState, t), t);
  k_set_state<<<(ctx->nbatch + 127) / 128, 128, 0, ctx->stream>>>(ctx->st, ctx->nbatch, offsetof(StepState, t_prev),
                                                                   t);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return DNSBOX_OK;
}

extern "C" int dnsbox_get_time(dnsbox_ctx *ctx, double *t) {
  BEGIN(ctx);
  if (!t) return set_err(DNSBOX_ERR_ARG, "null output");
  CK(cudaMemcpyAsync(ctx->hstage, &ctx->st->t, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *t = ctx->hstage[0];
  return DNSBOX_OK;
}

extern "C" int dnsbox_reset_history(dnsbox_ctx *ctx) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  ctx->ab2_started = 0;
  ctx->cfl_first = 1;
  return DNSBOX_OK;
}

// Internal: N(u) into out on the context's stream, with no device selection
// or host synchronisation (usable inside stream capture).
int rhs_nonlinear_impl(dnsbox_ctx *ctx, const void *uh, void *out) {
  return ctx->fp64 ? run_rhs<double>(ctx, uh, FIN_RHS, out, nullptr, nullptr, false, 0, nullptr)
                   : run_rhs<float>(ctx, uh, FIN_RHS, out, nullptr, nullptr, false, 0, nullptr);
}

extern "C" int dnsbox_rhs_nonlinear(dnsbox_ctx *ctx, const void *uh, void *out, double *eband) {
  BEGIN(ctx);
  if (!uh || !out) return set_err(DNSBOX_ERR_ARG, "null pointer");
  if (uh == out) return set_err(DNSBOX_ERR_ARG, "input and output may not alias");
  int rc = ctx->fp64 ? run_rhs<double>(ctx, uh, FIN_RHS, out, nullptr, nullptr, false, 0, nullptr)
                     : run_rhs<float>(ctx, uh, FIN_RHS, out, nullptr, nullptr, false, 0, nullptr);
  RET(rc);
  if (eband) {
    CK(cudaMemcpyAsync(ctx->hstage, &ctx->st->eband, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    RET(tc_check(ctx));
    *eband = ctx->p.bandlim ? ctx->hstage[0] : 0.0;
  }
  return DNSBOX_OK;
}

// Internal: decide pruning for state uh, then advance nsteps without further
// checks or diagnostics read-back (the trajectory of a state that vanishes on
// the cut set keeps vanishing there).  Used by the step-transpose chains.
int step_advance_decided(dnsbox_ctx *c, void *uh, int nsteps, bool decide) {
  if (decide) RET(c->fp64 ? prune_decide<double>(c, uh) : prune_decide<float>(c, uh));
  for (int n = 0; n < nsteps; ++n) RET(c->fp64 ? step_once<double>(c, uh) : step_once<float>(c, uh));
  return DNSBOX_OK;
}

extern "C" int dnsbox_step(dnsbox_ctx *ctx, void *uh, int nsteps, dnsbox_diag *diag) {
  BEGIN(ctx);
  if (!uh || nsteps < 0) return set_err(DNSBOX_ERR_ARG, "invalid argument");
  if (nsteps == 0) return DNSBOX_OK;
  return ctx->fp64 ? step_impl<double>(ctx, uh, nsteps, diag) : step_impl<float>(ctx, uh, nsteps, diag);
}

extern "C" int dnsbox_project(dnsbox_ctx *ctx, void *uh) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!uh) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const dnsbox_params &p = ctx->p;
  const int g = grid_for((long long)ctx->nh);
  if (ctx->fp64)
    k_project<double2><<<g, 256, 0, ctx->stream>>>((double2 *)uh, (long long)ctx->nh, p.nx, p.ny, p.nz,
                                                   p.alpha_x, p.alpha_y, p.alpha_z);
  else
    k_project<float2><<<g, 256, 0, ctx->stream>>>((float2 *)uh, (long long)ctx->nh, p.nx, p.ny, p.nz,
                                                  p.alpha_x, p.alpha_y, p.alpha_z);
  CK(cudaGetLastError());
  return DNSBOX_OK;
}

extern "C" int dnsbox_dealias(dnsbox_ctx *ctx, void *uh) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!uh) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const dnsbox_params &p = ctx->p;
  const int g = grid_for((long long)ctx->nh);
  const double cx = (p.nx / 2.0) * (2.0 * p.alpha_x / 3.0), cy = (p.ny / 2.0) * (2.0 * p.alpha_y / 3.0),
               cz = (p.nz / 2.0) * (2.0 * p.alpha_z / 3.0);
  const double sph2 = pow((p.nx / 2.0) * (2.0 * p.alpha_x / 3.0), 2);   // state.f90:189-190
  if (ctx->fp64)
    k_dealias<double2><<<g, 256, 0, ctx->stream>>>((double2 *)uh, (long long)ctx->nh, p.nx, p.ny, p.nz,
                                                   p.alpha_x, p.alpha_y, p.alpha_z, p.spherical, cx, cy,
                                                   cz, sph2);
  else
    k_dealias<float2><<<g, 256, 0, ctx->stream>>>((float2 *)uh, (long long)ctx->nh, p.nx, p.ny, p.nz,
                                                  p.alpha_x, p.alpha_y, p.alpha_z, p.spherical, cx, cy, cz,
                                                  sph2);
  CK(cudaGetLastError());
  return DNSBOX_OK;
}

// shared spectral diagnostics: out[0..nspec) spectrum, then ezero, eone, esqrt2, E-sum, D-sum
static int specdiag(dnsbox_ctx *ctx, const void *uh, int single, std::vector<double> &out) {
  const dnsbox_params &p = ctx->p;
  const int nv = ctx->nspec + 5;
  const int nblk = 148 * 2;
  RET(ensure_red(ctx, (size_t)nblk * nv + nv));
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  const size_t smem = (size_t)nv * sizeof(double);
  if (ctx->fp64)
    k_specdiag<double2><<<nblk, 256, smem, ctx->stream>>>((const double2 *)uh, (long long)ctx->nh, p.nx, p.ny,
                                                          p.nz, p.alpha_x, p.alpha_y, p.alpha_z, ctx->nspec,
                                                          p.Deltak, single, s * s, ctx->red);
  else
    k_specdiag<float2><<<nblk, 256, smem, ctx->stream>>>((const float2 *)uh, (long long)ctx->nh, p.nx, p.ny,
                                                         p.nz, p.alpha_x, p.alpha_y, p.alpha_z, ctx->nspec,
                                                         p.Deltak, single, s * s, ctx->red);
  CK(cudaGetLastError());
  k_sum_partials<<<(nv + 255) / 256, 256, 0, ctx->stream>>>(ctx->red, nblk, nv, ctx->red + (size_t)nblk * nv);
  CK(cudaGetLastError());
  out.resize(nv);
  CK(cudaMemcpyAsync(out.data(), ctx->red + (size_t)nblk * nv, nv * sizeof(double), cudaMemcpyDeviceToHost,
                     ctx->stream));
  RET(tc_check(ctx));
  return DNSBOX_OK;
}

extern "C" int dnsbox_spectrum(dnsbox_ctx *ctx, const void *uh, double *espec, double *ezero, double *eone,
                               double *esqrt2) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!uh) return set_err(DNSBOX_ERR_ARG, "null pointer");
  std::vector<double> v;
  RET(specdiag(ctx, uh, ctx->p.spectrum_mode == DNSBOX_SPECTRUM_SINGLE, v));
  const int ns = ctx->nspec;
  if (espec) memcpy(espec, v.data(), ns * sizeof(double));
  if (ezero) *ezero = v[ns];
  if (eone) *eone = v[ns + 1];
  if (esqrt2) *esqrt2 = v[ns + 2];
  return DNSBOX_OK;
}

extern "C" int dnsbox_kinetic(dnsbox_ctx *ctx, const void *uh, double *ekin) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!uh || !ekin) return set_err(DNSBOX_ERR_ARG, "null pointer");
  std::vector<double> v;
  RET(specdiag(ctx, uh, 0, v));
  const dnsbox_params &p = ctx->p;
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  *ekin = v[ctx->nspec + 3] * s * s;
  return DNSBOX_OK;
}

extern "C" int dnsbox_dissipation(dnsbox_ctx *ctx, const void *uh, double *disp) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!uh || !disp) return set_err(DNSBOX_ERR_ARG, "null pointer");
  std::vector<double> v;
  RET(specdiag(ctx, uh, 0, v));
  const dnsbox_params &p = ctx->p;
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  *disp = p.nu * v[ctx->nspec + 4] * s * s;
  return DNSBOX_OK;
}

extern "C" int dnsbox_eband(dnsbox_ctx *ctx, const void *uh, double *eband) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!uh || !eband) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const dnsbox_params &p = ctx->p;
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  if (!ctx->nband) {
    *eband = 0.0;
    return DNSBOX_OK;
  }
  if (ctx->fp64)
    k_eband<double2><<<1, 256, 0, ctx->stream>>>((const double2 *)uh, (long long)ctx->nh, ctx->band,
                                                 ctx->nband, p.nx, ctx->st, s * s, 0);
  else
    k_eband<float2><<<1, 256, 0, ctx->stream>>>((const float2 *)uh, (long long)ctx->nh, ctx->band, ctx->nband,
                                                p.nx, ctx->st, s * s, 0);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ctx->hstage, &ctx->st->eband, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *eband = ctx->hstage[0];
  return DNSBOX_OK;
}

// physical fields of the spectral state go to W1 (as 3 real fields after the
// z/y passes freed it); returns pointers to them.
template <typename T> static int state_to_phys(dnsbox_ctx *ctx, const void *uh, double scale, void **phys) {
  const void *in[3];
  void *out[3];
  // the c2r passes use W1 slots 0-2 and W2 slots 0-2; the physical output goes
  // to W1 slots 3-5 (each real field needs half a complex field's bytes)
  for (int f = 0; f < 3; ++f) {
    in[f] = cfield(reinterpret_cast<const char *>(uh), ctx, f);
    out[f] = field(ctx->W1, ctx, 3 + f);
    phys[f] = out[f];
  }
  return c2r_fields<T>(ctx, 3, in, out, scale);
}

static int reduce_max(dnsbox_ctx *ctx, const void *f, bool fp64, long long n, int absval, double *host) {
  const int nblk = 148 * 4;
  RET(ensure_red(ctx, nblk + 1));
  if (fp64)
    k_max<double><<<nblk, 256, 0, ctx->stream>>>((const double *)f, n, absval, ctx->red);
  else
    k_max<float><<<nblk, 256, 0, ctx->stream>>>((const float *)f, n, absval, ctx->red);
  CK(cudaGetLastError());
  k_max_partials<<<1, 1024, 0, ctx->stream>>>(ctx->red, nblk, ctx->red + nblk);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ctx->hstage, ctx->red + nblk, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  RET(tc_check(ctx));
  *host = ctx->hstage[0];
  return DNSBOX_OK;
}

extern "C" int dnsbox_courant(dnsbox_ctx *ctx, const void *uh, double dt, double *courant, double *umax3) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!uh || !courant) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const dnsbox_params &p = ctx->p;
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  void *phys[3];
  RET(ctx->fp64 ? state_to_phys<double>(ctx, uh, s, phys) : state_to_phys<float>(ctx, uh, s, phys));
  double m[3];
  for (int c = 0; c < 3; ++c) RET(reduce_max(ctx, phys[c], ctx->fp64, (long long)ctx->np, 1, &m[c]));
  // io.f90:669-671
  *courant = m[0] * dt / ((2 * M_PI / p.alpha_x) / p.nx) + m[1] * dt / ((2 * M_PI / p.alpha_y) / p.ny) +
             m[2] * dt / ((2 * M_PI / p.alpha_z) / p.nz);
  if (umax3)
    for (int c = 0; c < 3; ++c) umax3[c] = m[c];
  return DNSBOX_OK;
}

extern "C" int dnsbox_divergence(dnsbox_ctx *ctx, const void *uh, double *divmax) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!uh || !divmax) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const dnsbox_params &p = ctx->p;
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  // (i k . u) s into W2 slot 5, C2R into W1 slot 4
  void *dh = field(ctx->W2, ctx, 5);
  const int g = grid_for((long long)ctx->nh);
  if (ctx->fp64)
    k_divhat<double2><<<g, 256, 0, ctx->stream>>>((const double2 *)uh, (double2 *)dh, (long long)ctx->nh, p.nx,
                                                  p.ny, p.nz, p.alpha_x, p.alpha_y, p.alpha_z, s);
  else
    k_divhat<float2><<<g, 256, 0, ctx->stream>>>((const float2 *)uh, (float2 *)dh, (long long)ctx->nh, p.nx,
                                                 p.ny, p.nz, p.alpha_x, p.alpha_y, p.alpha_z, s);
  CK(cudaGetLastError());
  const void *in[1] = {dh};
  void *out[1] = {field(ctx->W1, ctx, 4)};
  RET(ctx->fp64 ? c2r_fields<double>(ctx, 1, in, out, 1.0) : c2r_fields<float>(ctx, 1, in, out, 1.0));
  return reduce_max(ctx, out[0], ctx->fp64, (long long)ctx->np, 0, divmax);
}

extern "C" int dnsbox_c2r(dnsbox_ctx *ctx, const void *spec, void *phys) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!spec || !phys) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const void *in[1] = {spec};
  void *out[1] = {phys};
  return ctx->fp64 ? c2r_fields<double>(ctx, 1, in, out, 1.0) : c2r_fields<float>(ctx, 1, in, out, 1.0);
}

extern "C" int dnsbox_r2c(dnsbox_ctx *ctx, const void *phys, void *spec) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!spec || !phys) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const void *in[1] = {phys};
  void *out[1] = {spec};
  return ctx->fp64 ? r2c_fields<double>(ctx, 1, in, out) : r2c_fields<float>(ctx, 1, in, out);
}

extern "C" int dnsbox_upload_state(dnsbox_ctx *ctx, const double *host, void *uh) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!host || !uh) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const dnsbox_params &p = ctx->p;
  // 3 complex-double fields fit in W1 (6 fields of the context precision >= 3 x 16 B)
  const size_t bytes = 3 * ctx->nh * 16;
  CK(cudaMemcpyAsync(ctx->W1, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
  dim3 grid((p.nz + 31) / 32, (ctx->nxh + 31) / 32, 3 * p.ny), blk(32, 8);
  if (ctx->fp64)
    k_from_p3dfft<double2><<<grid, blk, 0, ctx->stream>>>((const double2 *)ctx->W1, (double2 *)uh, ctx->nxh,
                                                          p.ny, p.nz);
  else
    k_from_p3dfft<float2><<<grid, blk, 0, ctx->stream>>>((const double2 *)ctx->W1, (float2 *)uh, ctx->nxh, p.ny,
                                                         p.nz);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return DNSBOX_OK;
}

extern "C" int dnsbox_download_state(dnsbox_ctx *ctx, const void *uh, double *host) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!host || !uh) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const dnsbox_params &p = ctx->p;
  dim3 grid((p.nz + 31) / 32, (ctx->nxh + 31) / 32, 3 * p.ny), blk(32, 8);
  if (ctx->fp64)
    k_to_p3dfft<double2><<<grid, blk, 0, ctx->stream>>>((const double2 *)uh, (double2 *)ctx->W1, ctx->nxh, p.ny,
                                                        p.nz);
  else
    k_to_p3dfft<float2><<<grid, blk, 0, ctx->stream>>>((const float2 *)uh, (double2 *)ctx->W1, ctx->nxh, p.ny,
                                                       p.nz);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, ctx->W1, 3 * ctx->nh * 16, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return DNSBOX_OK;
}

extern "C" int dnsbox_upload_physical(dnsbox_ctx *ctx, const double *host, void *uh) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!host || !uh) return set_err(DNSBOX_ERR_ARG, "null pointer");
  // host doubles -> W2 (3 physical double fields fit: 6 nh cbytes >= 3 np 8 for both precisions)
  const size_t pbytes = ctx->np * sizeof(double);
  CK(cudaMemcpyAsync(ctx->W2, host, 3 * pbytes, cudaMemcpyHostToDevice, ctx->stream));
  const void *in[3];
  void *out[3];
  char *src = ctx->W2;
  if (!ctx->fp64) {
    // convert to float into W1 slots 3-5 (each holds nh*8 B >= np*4 B)
    for (int c = 0; c < 3; ++c) {
      float *dst = reinterpret_cast<float *>(field(ctx->W1, ctx, 3 + c));
      k_convert<double, float><<<grid_for((long long)ctx->np), 256, 0, ctx->stream>>>(
          reinterpret_cast<const double *>(src + c * pbytes), dst, (long long)ctx->np);
      in[c] = dst;
    }
    CK(cudaGetLastError());
  } else {
    for (int c = 0; c < 3; ++c) in[c] = src + c * pbytes;
  }
  for (int c = 0; c < 3; ++c) out[c] = field(reinterpret_cast<char *>(uh), ctx, c);
  RET(ctx->fp64 ? r2c_fields<double>(ctx, 3, in, out) : r2c_fields<float>(ctx, 3, in, out));
  RET(tc_check(ctx));
  return DNSBOX_OK;
}

// 3D R2C of three physical fields of the context precision (3 np elements at
// phys; may live in W2, which the x-line pass consumes before it is reused).
template <typename T> static int phys3_to_state(dnsbox_ctx *ctx, const void *phys, void *uh) {
  const void *in[3];
  void *out[3];
  for (int c = 0; c < 3; ++c) {
    in[c] = reinterpret_cast<const T *>(phys) + (size_t)c * ctx->np;
    out[c] = field(reinterpret_cast<char *>(uh), ctx, c);
  }
  return r2c_fields<T>(ctx, 3, in, out);
}

extern "C" int dnsbox_init_yoffe(dnsbox_ctx *ctx, const void *noise3_dev, uint64_t seed, void *uh) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!uh) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const dnsbox_params &p = ctx->p;
  const void *noise = noise3_dev;
  if (!noise) {   // intent of state.f90:231-236: all three components uniform in [-0.5, 0.5)
    const long long n3 = 3 * (long long)ctx->np;
    if (ctx->fp64) k_noise<double><<<grid_for(n3), 256, 0, ctx->stream>>>((double *)ctx->W2, n3, seed);
    else k_noise<float><<<grid_for(n3), 256, 0, ctx->stream>>>((float *)ctx->W2, n3, seed);
    CK(cudaGetLastError());
    noise = ctx->W2;
  }
  RET(ctx->fp64 ? phys3_to_state<double>(ctx, noise, uh) : phys3_to_state<float>(ctx, noise, uh));   // :240
  RET(dnsbox_dealias(ctx, uh));   // :242
  RET(dnsbox_project(ctx, uh));   // :243
  std::vector<double> v;          // :244 (state_spectrum, in the context's spectrum mode)
  RET(specdiag(ctx, uh, p.spectrum_mode == DNSBOX_SPECTRUM_SINGLE, v));
  const int ns = ctx->nspec;
  RET(ensure_red(ctx, (size_t)ns));
  CK(cudaMemcpyAsync(ctx->red, v.data(), ns * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  const long long nh = (long long)ctx->nh;
  if (ctx->fp64)
    k_yoffe_rescale<double2><<<grid_for(nh), 256, 0, ctx->stream>>>((double2 *)uh, nh, p.nx, p.ny, p.nz, p.alpha_x,
                                                                    p.alpha_y, p.alpha_z, p.Deltak, ns, ctx->red);
  else
    k_yoffe_rescale<float2><<<grid_for(nh), 256, 0, ctx->stream>>>((float2 *)uh, nh, p.nx, p.ny, p.nz, p.alpha_x,
                                                                   p.alpha_y, p.alpha_z, p.Deltak, ns, ctx->red);
  CK(cudaGetLastError());
  RET(tc_check(ctx));   // the host vector v is read by the copy above before it goes out of scope
  return DNSBOX_OK;
}

extern "C" int dnsbox_init_beltrami(dnsbox_ctx *ctx, double t, void *uh) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!uh) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const dnsbox_params &p = ctx->p;
  const double lx = 2 * M_PI / p.alpha_x, ly = 2 * M_PI / p.alpha_y, lz = 2 * M_PI / p.alpha_z;
  const long long np = (long long)ctx->np;
  if (ctx->fp64)
    k_beltrami<double><<<grid_for(np), 256, 0, ctx->stream>>>((double *)ctx->W2, p.nx, p.ny, p.nz, lx, ly, lz, p.nu, t);
  else
    k_beltrami<float><<<grid_for(np), 256, 0, ctx->stream>>>((float *)ctx->W2, p.nx, p.ny, p.nz, lx, ly, lz, p.nu, t);
  CK(cudaGetLastError());
  RET(ctx->fp64 ? phys3_to_state<double>(ctx, ctx->W2, uh) : phys3_to_state<float>(ctx, ctx->W2, uh));
  RET(tc_check(ctx));
  return DNSBOX_OK;
}

extern "C" int dnsbox_set_step_projection(dnsbox_ctx *ctx, int on) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  ctx->proj_every = on ? 1 : 0;
  return DNSBOX_OK;
}

extern "C" int dnsbox_download_physical(dnsbox_ctx *ctx, const void *uh, double *host) {
  BEGIN(ctx);
  SINGLE(ctx);
  if (!host || !uh) return set_err(DNSBOX_ERR_ARG, "null pointer");
  const dnsbox_params &p = ctx->p;
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  void *phys[3];
  RET(ctx->fp64 ? state_to_phys<double>(ctx, uh, s, phys) : state_to_phys<float>(ctx, uh, s, phys));
  const size_t pbytes = ctx->np * sizeof(double);
  for (int c = 0; c < 3; ++c) {
    if (ctx->fp64) {
      CK(cudaMemcpyAsync(reinterpret_cast<char *>(host) + c * pbytes, phys[c], pbytes, cudaMemcpyDeviceToHost,
                         ctx->stream));
    } else {
      double *stage = reinterpret_cast<double *>(ctx->W2);   // free after the c2r passes
      k_convert<float, double><<<grid_for((long long)ctx->np), 256, 0, ctx->stream>>>(
          reinterpret_cast<const float *>(phys[c]), stage, (long long)ctx->np);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(reinterpret_cast<char *>(host) + c * pbytes, stage, pbytes, cudaMemcpyDeviceToHost,
                         ctx->stream));
    }
  }
  RET(tc_check(ctx));
  return DNSBOX_OK;
}


extern "C" int dnsbox_sync(dnsbox_ctx *ctx) {
  BEGIN(ctx);
  return tc_check(ctx);
}

extern "C" int dnsbox_profile_enable(dnsbox_ctx *ctx, int on) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  ctx->prof_on = on ? 1 : 0;
  return DNSBOX_OK;
}

extern "C" int dnsbox_profile_read(dnsbox_ctx *ctx, dnsbox_profile *out, int reset) {
  BEGIN(ctx);
  if (!out) return set_err(DNSBOX_ERR_ARG, "null output");
  CK(cudaStreamSynchronize(ctx->stream));
  memset(out, 0, sizeof(*out));
  for (size_t i = 0; i < ctx->ev_used; ++i) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev_pool[2 * i], ctx->ev_pool[2 * i + 1]));
    out->ms[ctx->ev_kind[i]] += ms;
  }
  for (int k = 0; k < DNSBOX_NPASS; ++k) out->launches[k] = ctx->launches[k];
  out->total_launches = ctx->total_launches;
  if (reset) {
    ctx->ev_used = 0;
    for (int k = 0; k < DNSBOX_NPASS; ++k) ctx->launches[k] = 0;
    ctx->total_launches = 0;
  }
  return DNSBOX_OK;
}

extern "C" int dnsbox_set_forcing(dnsbox_ctx *ctx, const void *f3_dev) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  ctx->force = f3_dev;
  return DNSBOX_OK;
}

extern "C" int dnsbox_state_alloc(dnsbox_ctx *ctx, void **out) {
  BEGIN(ctx);
  if (!out) return set_err(DNSBOX_ERR_ARG, "null output");
  *out = nullptr;
  CK(cudaMalloc(out, 3 * ctx->nh * ctx->cbytes));
  CK(cudaMemset(*out, 0, 3 * ctx->nh * ctx->cbytes));
  return DNSBOX_OK;
}

extern "C" int dnsbox_state_free(dnsbox_ctx *ctx, void *p) {
  BEGIN(ctx);
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaFree(p));
  return DNSBOX_OK;
}

extern "C" int dnsbox_set_batch_nu(dnsbox_ctx *ctx, const double *nu_host) {
  BEGIN(ctx);
  if (!nu_host) return set_err(DNSBOX_ERR_ARG, "null pointer");
  for (int b = 0; b < ctx->nbatch; ++b)
    if (!(nu_host[b] >= 0.0)) return set_err(DNSBOX_ERR_ARG, "invalid viscosity for box %d", b);
  if (ctx->nbatch == 1) {
    ctx->p.nu = nu_host[0];
    return DNSBOX_OK;
  }
  CK(cudaMemcpy(ctx->d_nu, nu_host, ctx->nbatch * sizeof(double), cudaMemcpyHostToDevice));
  return DNSBOX_OK;
}

extern "C" int dnsbox_diag_read(dnsbox_ctx *ctx, int nrecent, dnsbox_diag *host) {
  BEGIN(ctx);
  if (!host || nrecent < 0) return set_err(DNSBOX_ERR_ARG, "invalid argument");
  if (nrecent > ctx->ring_cap || nrecent > ctx->host_step)
    return set_err(DNSBOX_ERR_ARG, "only the last %d steps are kept (%lld issued)", ctx->ring_cap,
                   (long long)ctx->host_step);
  return ring_read(ctx, ctx->host_step - nrecent, nrecent, host);
}

extern "C" int dnsbox_batch_size(const dnsbox_ctx *ctx) { return ctx ? ctx->nbatch : -1; }

// ------------------------------------------------------------------ ensemble
// The graphs are captured and replayed on a private stream (the legacy
// default stream cannot be captured); events order them after the contexts'
// stream on entry and make that stream wait for them on exit.  Two graphs:
// the full passes, and (when every context allows it) the pruned passes,
// which a replay may use while every state vanishes on its 2/3-rule cut set
// -- the steps keep it so, and dnsbox_ensemble_run checks it once per call.
struct dnsbox_ensemble {
  std::vector<dnsbox_ctx *> ctxs;
  std::vector<void *> states;
  cudaStream_t user = 0, own = nullptr;
  cudaEvent_t in = nullptr, out = nullptr;
  cudaGraph_t graph[2] = {nullptr, nullptr};   // [0] full passes, [1] pruned passes
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  int last_pruned = 0;
  // capture: one branch stream per context, forked from and joined into `own`,
  // so that the graph runs the contexts' steps as independent branches
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr;
};

static int step_any(dnsbox_ctx *c, void *u) {
  return c->fp64 ? step_once<double>(c, u) : step_once<float>(c, u);
}

static int prune_decide_any(dnsbox_ctx *c, void *u) {
  return c->fp64 ? prune_decide<double>(c, u) : prune_decide<float>(c, u);
}

static int cut_check_any(dnsbox_ctx *c, void *u) {
  return c->fp64 ? cut_check_async<double>(c, u) : cut_check_async<float>(c, u);
}

static void ensemble_free(dnsbox_ensemble *e) {
  if (!e) return;
  if (e->own) cudaStreamSynchronize(e->own);
  for (int g = 0; g < 2; ++g) {
    if (e->exec[g]) cudaGraphExecDestroy(e->exec[g]);
    if (e->graph[g]) cudaGraphDestroy(e->graph[g]);
  }
  if (e->in) cudaEventDestroy(e->in);
  if (e->out) cudaEventDestroy(e->out);
  if (e->fork) cudaEventDestroy(e->fork);
  for (cudaEvent_t j : e->joins)
    if (j) cudaEventDestroy(j);
  for (cudaStream_t b : e->branch)
    if (b) cudaStreamDestroy(b);
  if (e->own) cudaStreamDestroy(e->own);
  for (auto *c : e->ctxs) {
    c->stream = e->user;
    c->prune_now = 0;
  }
  delete e;
}

// Captures one step of every context (pruned passes where `pruned`) into
// e->graph[g] / e->exec[g].
static int ensemble_capture(dnsbox_ensemble *e, int g, bool pruned) {
  const int n = (int)e->ctxs.size();
  for (auto *c : e->ctxs) {
    c->stream = e->own;
    c->prune_now = pruned ? 1 : 0;
  }
  CK(cudaStreamBeginCapture(e->own, cudaStreamCaptureModeThreadLocal));
  int rc = DNSBOX_OK;
  cudaError_t cerr = cudaEventRecord(e->fork, e->own);
  for (int i = 0; i < n && rc == DNSBOX_OK && cerr == cudaSuccess; ++i) {
    if ((cerr = cudaStreamWaitEvent(e->branch[i], e->fork, 0)) != cudaSuccess) break;
    e->ctxs[i]->stream = e->branch[i];
    rc = step_any(e->ctxs[i], e->states[i]);
    if (rc == DNSBOX_OK && (cerr = cudaEventRecord(e->joins[i], e->branch[i])) == cudaSuccess)
      cerr = cudaStreamWaitEvent(e->own, e->joins[i], 0);
  }
  if (rc == DNSBOX_OK && cerr != cudaSuccess) rc = set_err(DNSBOX_ERR_CUDA, "ensemble capture: %s", cudaGetErrorString(cerr));
  const cudaError_t err = cudaStreamEndCapture(e->own, &e->graph[g]);
  for (auto *c : e->ctxs) {
    c->host_step -= 1;   // the captured step has not run
    c->stream = e->user;
    c->prune_now = 0;
  }
  if (rc != DNSBOX_OK) return rc;
  if (err != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(err));
  CK(cudaGraphInstantiate(&e->exec[g], e->graph[g], 0));
  return DNSBOX_OK;
}

extern "C" int dnsbox_ensemble_create(dnsbox_ctx *const *ctxs, void *const *states, int n, dnsbox_ensemble **out) {
  if (!ctxs || !states || !out || n <= 0) return set_err(DNSBOX_ERR_ARG, "invalid argument");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i] || !states[i]) return set_err(DNSBOX_ERR_ARG, "null context or state %d", i);
    if (ctxs[i]->p.device != ctxs[0]->p.device) return set_err(DNSBOX_ERR_ARG, "contexts on different devices");
    if (ctxs[i]->prof_on) return set_err(DNSBOX_ERR_STATE, "profiling must be off while capturing");
    if (ctxs[i]->p.stepper == DNSBOX_SEMI_IMPLICIT)
      return set_err(DNSBOX_ERR_UNSUPPORTED, "the semi-implicit step reads its iterations back: not capturable");
  }
  CK(cudaSetDevice(ctxs[0]->p.device));
  dnsbox_ensemble *e = new dnsbox_ensemble();
  e->ctxs.assign(ctxs, ctxs + n);
  e->states.assign(states, states + n);
  e->user = ctxs[0]->stream;
  auto fail = [&](cudaError_t err, const char *what) {
    ensemble_free(e);
    return set_err(DNSBOX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(err));
  };
  auto fail_rc = [&](int rc) {
    ensemble_free(e);
    return rc;
  };
  cudaError_t err;
  if ((err = cudaStreamCreateWithFlags(&e->own, cudaStreamNonBlocking)) != cudaSuccess) return fail(err, "stream");
  if ((err = cudaEventCreateWithFlags(&e->in, cudaEventDisableTiming)) != cudaSuccess) return fail(err, "event");
  if ((err = cudaEventCreateWithFlags(&e->out, cudaEventDisableTiming)) != cudaSuccess) return fail(err, "event");
  if ((err = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming)) != cudaSuccess) return fail(err, "event");
  e->branch.assign(n, nullptr);
  e->joins.assign(n, nullptr);
  for (int i = 0; i < n; ++i) {
    if ((err = cudaStreamCreateWithFlags(&e->branch[i], cudaStreamNonBlocking)) != cudaSuccess) return fail(err, "stream");
    if ((err = cudaEventCreateWithFlags(&e->joins[i], cudaEventDisableTiming)) != cudaSuccess) return fail(err, "event");
  }
  for (auto *c : e->ctxs) c->stream = e->user;
  // one eager step on the contexts' stream, so the captured step is a steady
  // one (the first step's forced dt update and the AB2 start-up are host-side
  // decisions); it decides pruning per context as dnsbox_step does
  bool all_pruned = true;
  for (int i = 0; i < n; ++i) {
    int rc = prune_decide_any(e->ctxs[i], e->states[i]);
    if (rc == DNSBOX_OK) rc = step_any(e->ctxs[i], e->states[i]);
    if (rc != DNSBOX_OK) return fail_rc(rc);
    all_pruned = all_pruned && e->ctxs[i]->prune_now;
    e->ctxs[i]->prune_now = 0;
  }
  if ((err = cudaEventRecord(e->in, e->user)) != cudaSuccess) return fail(err, "event record");
  if ((err = cudaStreamWaitEvent(e->own, e->in, 0)) != cudaSuccess) return fail(err, "stream wait");
  int rc = ensemble_capture(e, 0, false);
  if (rc == DNSBOX_OK && all_pruned) rc = ensemble_capture(e, 1, true);
  if (rc != DNSBOX_OK) return fail_rc(rc);
  *out = e;
  return DNSBOX_OK;
}

// The pruned graph when every state still vanishes on its cut set (one check
// kernel per context and one 4-byte read per call), else the full graph.
extern "C" int dnsbox_ensemble_run(dnsbox_ensemble *e, int nsteps) {
  if (!e || nsteps < 0) return set_err(DNSBOX_ERR_ARG, "invalid argument");
  CK(cudaSetDevice(e->ctxs[0]->p.device));
  int g = 0;
  if (e->exec[1] && nsteps > 0) {
    const int n = (int)e->ctxs.size();
    for (int i = 0; i < n; ++i) {
      dnsbox_ctx *c = e->ctxs[i];
      RET(cut_check_any(c, e->states[i]));   // on the user stream, after the caller's work
    }
    // each context's check writes its own flag; they are folded on the host
    int clean = 1;
    for (int i = 0; i < n; ++i) {
      dnsbox_ctx *c = e->ctxs[i];
      int *flag = reinterpret_cast<int *>(c->hstage + 62);
      CK(cudaMemcpyAsync(flag, c->cut_flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(e->user));
    for (int i = 0; i < n; ++i) clean = clean && *reinterpret_cast<int *>(e->ctxs[i]->hstage + 62) == 0;
    g = clean ? 1 : 0;
  }
  e->last_pruned = g;
  CK(cudaEventRecord(e->in, e->user));
  CK(cudaStreamWaitEvent(e->own, e->in, 0));
  for (int i = 0; i < nsteps; ++i) {
    CK(cudaGraphLaunch(e->exec[g], e->own));
    for (auto *c : e->ctxs) c->host_step += 1;
  }
  CK(cudaEventRecord(e->out, e->own));
  CK(cudaStreamWaitEvent(e->user, e->out, 0));
  return DNSBOX_OK;
}

extern "C" int dnsbox_ensemble_pruned(const dnsbox_ensemble *e) { return e ? e->last_pruned : -1; }

extern "C" int dnsbox_ensemble_destroy(dnsbox_ensemble *e) {
  if (!e) return DNSBOX_OK;
  cudaSetDevice(e->ctxs[0]->p.device);
  ensemble_free(e);
  return DNSBOX_OK;
}
