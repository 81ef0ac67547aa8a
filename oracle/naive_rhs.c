/* Naive-DFT restatement of dnsbox's rhs_nonlinear -- TEST INFRASTRUCTURE ONLY.
 *
 * An independent cross-check of the NumPy oracle's transform conventions
 * (sign, unnormalised scaling, half-spectrum layout, C2R treatment of the kx = 0
 * and Nyquist bins, Nyquist wavenumbers set to zero) for grids of a few points.
 * Every transform is a separable direct DFT with twiddles evaluated in long
 * double from the exact integer phase (k*n mod N)/N; no FFT algorithm is used.
 *
 * Restates rhs.f90:18-135 (rotational form; 9 + 3 C2R, 3 R2C, spectral loop
 * with the 2/3 mask, pressure projection and band forcing), rhs_Eband
 * (rhs.f90:137-168) and the wavenumber tables of variables.f90:226-262.
 *
 * Layout: spectral [3][nz][ny][nx/2+1] interleaved complex double (kx
 * fastest); physical [nz][ny][nx] double (x fastest).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cpx;

static const long double TWO_PI_L = 6.283185307179586476925286766559005768L;

static cpx cexp_idx(long long k, long long n, int len, int sign) {
  long long m = ((k * n) % len + len) % len;
  long double a = TWO_PI_L * (long double)m / (long double)len;
  cpx r = {(double)cosl(a), (double)(sign * sinl(a))};
  return r;
}

static double k_full(int idx, int n, double alpha) {       /* variables.f90:242-262 */
  if (idx == n / 2) return 0.0;
  return (idx < n / 2 ? idx : idx - n) * alpha;
}
static double k_half(int idx, int n, double alpha) {       /* variables.f90:226-233 */
  return idx == n / 2 ? 0.0 : idx * alpha;
}

/* half spectrum F[nz][ny][nxh] -> real f[nz][ny][nx], unnormalised */
static void naive_c2r(int nx, int ny, int nz, const cpx *F, double *f) {
  int nxh = nx / 2 + 1;
  size_t nh = (size_t)nz * ny * nxh;
  cpx *a = malloc(nh * sizeof(cpx)), *b = malloc(nh * sizeof(cpx));
  for (int z = 0; z < nz; ++z)
    for (int ky = 0; ky < ny; ++ky)
      for (int kx = 0; kx < nxh; ++kx) {
        long double sr = 0, si = 0;
        for (int kz = 0; kz < nz; ++kz) {
          cpx w = cexp_idx(kz, z, nz, +1), v = F[((size_t)kz * ny + ky) * nxh + kx];
          sr += (long double)v.re * w.re - (long double)v.im * w.im;
          si += (long double)v.re * w.im + (long double)v.im * w.re;
        }
        a[((size_t)z * ny + ky) * nxh + kx] = (cpx){(double)sr, (double)si};
      }
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int kx = 0; kx < nxh; ++kx) {
        long double sr = 0, si = 0;
        for (int ky = 0; ky < ny; ++ky) {
          cpx w = cexp_idx(ky, y, ny, +1), v = a[((size_t)z * ny + ky) * nxh + kx];
          sr += (long double)v.re * w.re - (long double)v.im * w.im;
          si += (long double)v.re * w.im + (long double)v.im * w.re;
        }
        b[((size_t)z * ny + y) * nxh + kx] = (cpx){(double)sr, (double)si};
      }
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const cpx *row = b + ((size_t)z * ny + y) * nxh;
        long double s = row[0].re;
        if (nx % 2 == 0) s += (long double)row[nx / 2].re * ((x % 2) ? -1.0L : 1.0L);
        int kmax = (nx % 2 == 0) ? nx / 2 - 1 : nx / 2;
        for (int k = 1; k <= kmax; ++k) {
          cpx w = cexp_idx(k, x, nx, +1);
          s += 2.0L * ((long double)row[k].re * w.re - (long double)row[k].im * w.im);
        }
        f[((size_t)z * ny + y) * nx + x] = (double)s;
      }
  free(a);
  free(b);
}

/* real f[nz][ny][nx] -> half spectrum F, unnormalised */
static void naive_r2c(int nx, int ny, int nz, const double *f, cpx *F) {
  int nxh = nx / 2 + 1;
  size_t nh = (size_t)nz * ny * nxh;
  cpx *a = malloc(nh * sizeof(cpx)), *b = malloc(nh * sizeof(cpx));
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int k = 0; k < nxh; ++k) {
        long double sr = 0, si = 0;
        for (int x = 0; x < nx; ++x) {
          cpx w = cexp_idx(k, x, nx, -1);
          double v = f[((size_t)z * ny + y) * nx + x];
          sr += (long double)v * w.re;
          si += (long double)v * w.im;
        }
        a[((size_t)z * ny + y) * nxh + k] = (cpx){(double)sr, (double)si};
      }
  for (int z = 0; z < nz; ++z)
    for (int ky = 0; ky < ny; ++ky)
      for (int k = 0; k < nxh; ++k) {
        long double sr = 0, si = 0;
        for (int y = 0; y < ny; ++y) {
          cpx w = cexp_idx(ky, y, ny, -1), v = a[((size_t)z * ny + y) * nxh + k];
          sr += (long double)v.re * w.re - (long double)v.im * w.im;
          si += (long double)v.re * w.im + (long double)v.im * w.re;
        }
        b[((size_t)z * ny + ky) * nxh + k] = (cpx){(double)sr, (double)si};
      }
  for (int kz = 0; kz < nz; ++kz)
    for (int ky = 0; ky < ny; ++ky)
      for (int k = 0; k < nxh; ++k) {
        long double sr = 0, si = 0;
        for (int z = 0; z < nz; ++z) {
          cpx w = cexp_idx(kz, z, nz, -1), v = b[((size_t)z * ny + ky) * nxh + k];
          sr += (long double)v.re * w.re - (long double)v.im * w.im;
          si += (long double)v.re * w.im + (long double)v.im * w.re;
        }
        F[((size_t)kz * ny + ky) * nxh + k] = (cpx){(double)sr, (double)si};
      }
  free(a);
  free(b);
}

int naive_c2r_field(int nx, int ny, int nz, const double *spec, double *phys) {
  naive_c2r(nx, ny, nz, (const cpx *)spec, phys);
  return 0;
}

int naive_r2c_field(int nx, int ny, int nz, const double *phys, double *spec) {
  naive_r2c(nx, ny, nz, phys, (cpx *)spec);
  return 0;
}

/* prm: alpha_x, alpha_y, alpha_z, nu, Q, Pin, kCutOff, bandlim, spherical */
int naive_rhs_nonlinear(int nx, int ny, int nz, const double *prm, const double *uhat_in,
                        double *out_in, double *eband_out) {
  const double ax = prm[0], ay = prm[1], az = prm[2];
  const double Pin = prm[5], kcut = prm[6];
  const int bandlim = prm[7] != 0.0, spherical = prm[8] != 0.0;
  const int nxh = nx / 2 + 1;
  const size_t nh = (size_t)nz * ny * nxh, np = (size_t)nz * ny * nx;
  const double s = 1.0 / ((double)nx * ny * nz);
  const cpx *uh = (const cpx *)uhat_in;
  cpx *out = (cpx *)out_in;

  /* rhs_Eband (rhs.f90:137-168) */
  double eband = 0.0;
  if (bandlim) {
    for (int kz = 0; kz < nz; ++kz)
      for (int ky = 0; ky < ny; ++ky)
        for (int kx = 0; kx < nxh; ++kx) {
          double kxr = k_half(kx, nx, ax), kyr = k_full(ky, ny, ay), kzr = k_full(kz, nz, az);
          double absk = sqrt(kxr * kxr + kyr * kyr + kzr * kzr);
          if (absk > kcut) continue;
          double sc = (kxr == 0.0) ? 0.5 : 1.0;
          size_t i = ((size_t)kz * ny + ky) * nxh + kx;
          for (int c = 0; c < 3; ++c) {
            cpx v = uh[c * nh + i];
            eband += (v.re * v.re + v.im * v.im) * sc;
          }
        }
    eband *= s * s;
  }
  if (eband_out) *eband_out = eband;

  /* derivatives (state.f90:456-500), vorticity (state.f90:502-515) */
  cpx *tc = malloc(nh * sizeof(cpx));
  double *d = malloc(9 * np * sizeof(double));
  for (int ci = 0; ci < 3; ++ci)
    for (int j = 0; j < 3; ++j) {
      for (int kz = 0; kz < nz; ++kz)
        for (int ky = 0; ky < ny; ++ky)
          for (int kx = 0; kx < nxh; ++kx) {
            double kr = j == 0 ? k_half(kx, nx, ax) : j == 1 ? k_full(ky, ny, ay) : k_full(kz, nz, az);
            size_t i = ((size_t)kz * ny + ky) * nxh + kx;
            cpx v = uh[ci * nh + i];
            /* uhat * (i k) * scalemodes */
            tc[i] = (cpx){-v.im * kr * s, v.re * kr * s};
          }
      naive_c2r(nx, ny, nz, tc, d + (size_t)(3 * ci + j) * np);
    }
#define D(i, j) (d + (size_t)(3 * (i) + (j)) * np)
  double *om = malloc(3 * np * sizeof(double)), *ut = malloc(3 * np * sizeof(double));
  for (size_t p = 0; p < np; ++p) {
    om[p] = D(2, 1)[p] - D(1, 2)[p];
    om[np + p] = D(0, 2)[p] - D(2, 0)[p];
    om[2 * np + p] = D(1, 0)[p] - D(0, 1)[p];
  }
  for (int c = 0; c < 3; ++c) naive_c2r(nx, ny, nz, uh + c * nh, ut + c * np);
  double *tr = malloc(np * sizeof(double));
  cpx *nl = malloc(3 * nh * sizeof(cpx));
  for (int c = 0; c < 3; ++c) {
    for (size_t p = 0; p < np; ++p) {
      double ox = om[p], oy = om[np + p], oz = om[2 * np + p];
      double u = ut[p], v = ut[np + p], w = ut[2 * np + p];
      double val = c == 0 ? oy * w - oz * v : c == 1 ? oz * u - ox * w : ox * v - oy * u;
      tr[p] = val * s;
    }
    naive_r2c(nx, ny, nz, tr, nl + c * nh);
  }
  /* spectral loop (rhs.f90:67-133) */
  const double cx = (nx / 2.0) * (2.0 * ax / 3.0), cy = (ny / 2.0) * (2.0 * ay / 3.0),
               cz = (nz / 2.0) * (2.0 * az / 3.0);
  for (int kz = 0; kz < nz; ++kz)
    for (int ky = 0; ky < ny; ++ky)
      for (int kx = 0; kx < nxh; ++kx) {
        size_t i = ((size_t)kz * ny + ky) * nxh + kx;
        double kr[3] = {k_half(kx, nx, ax), k_full(ky, ny, ay), k_full(kz, nz, az)};
        double k2 = kr[0] * kr[0] + kr[1] * kr[1] + kr[2] * kr[2];
        double absk = sqrt(k2);
        int zero = kr[0] == 0.0 && kr[1] == 0.0 && kr[2] == 0.0;
        int cut = (spherical && k2 >= pow((nx / 2.0) * 0.5 * ax, 2)) || fabs(kr[0]) >= cx ||
                  fabs(kr[1]) >= cy || fabs(kr[2]) >= cz || zero;
        if (cut) {
          for (int c = 0; c < 3; ++c) out[c * nh + i] = (cpx){0.0, 0.0};
          continue;
        }
        /* phat = -(i k . n) / (-(k.k)) = i (k.n) / |k|^2 */
        double kn_re = 0, kn_im = 0;
        for (int c = 0; c < 3; ++c) {
          cpx n = nl[c * nh + i];
          kn_re += kr[c] * n.re;
          kn_im += kr[c] * n.im;
        }
        cpx phat = {-kn_im / k2, kn_re / k2};
        double fc = (bandlim && absk <= kcut) ? Pin / (2.0 * eband) : 0.0;
        for (int c = 0; c < 3; ++c) {
          cpx n = nl[c * nh + i], u = uh[c * nh + i];
          /* -n - (i k_c) phat + fc u */
          double re = -n.re + kr[c] * phat.im + fc * u.re;
          double im = -n.im - kr[c] * phat.re + fc * u.im;
          out[c * nh + i] = (cpx){re, im};
        }
      }
#undef D
  free(tc);
  free(d);
  free(om);
  free(ut);
  free(tr);
  free(nl);
  return 0;
}
