// Adjoint operators and adjoint descent.
//
//  dnsbox_rhs_adj            rhsAdj (rhsAdj.f90:356-381), restated literally:
//                            convective-form N (rhsAdj.f90:64-175, '.gt.' mask,
//                            eps = 1e-13 at k = 0), r~ = H^-1 (L u + N)
//                            (rhsupptilde, :177-213), the adjoint nonlinear term
//                            -P_d[(grad r~)^T u + (u.grad) r~] (:261-354) and
//                            rhsadj = L r~ + N_adj.
//  dnsbox_rhs_nonlinear_vjp  the exact transpose of the linearised
//                            rhs_nonlinear (Euclidean inner product on the Re/Im
//                            parts of the half spectrum):
//                              h = -P(D g),  phi = C2R(h / W),
//                              u = C2R(uhat) s,  omega = C2R(ik x uhat) s,
//                              out = s W (ik x R2C(u x phi) + R2C(phi x omega))
//                            plus the band-forcing term when bandlim is on.
//  dnsbox_residual(_grad)    J = 1/2 s^2 sum_half W h |r|^2 with r = L u + N(u) + f
//                            (h = 1/(1+|k|^2) when hminone), and its gradient.
//  dnsbox_adjoint_descent    steepest descent on J with an FP64 Armijo line search.
//  dnsbox_heun_step_vjp      transpose of one fixed-dt IF-Heun step
//                              S(u) = IF u + dt/2 IF N(u) + dt/2 N(u*), u* = IF (u + dt N(u)):
//                              a = N'(u*)^T (dt/2 g),
//                              S'(u)^T g = IF (g + a) + N'(u)^T (IF (dt/2 g + dt a)).
//  dnsbox_heun_steps_vjp     the transpose of nsteps such steps, with the states
//                            recomputed per segment from checkpoints taken every
//                            `every` steps (memory: nsteps/every + every states).
//  dnsbox_orbit_residual     J = 1/2 <(u(T) - u(0))^2> (physical mean square) of the
//                            periodic-orbit problem and its gradient (Phi'^T - I)(s^2 W r).
//
// W is the half-spectrum multiplicity (1 on the kx = 0 and Nyquist planes, 2
// elsewhere); L = Q - nu |k|^2 (the reference's nu (k.k) + Q with imaginary k).
#include <memory>

#include "internal.cuh"

namespace {

struct Grid3 {
  int nx, ny, nz, nxh;
  double ax, ay, az;
  double cutx, cuty, cutz, sph2;
  int spherical;
};

__device__ __forceinline__ void mode_k(const Grid3 &g, long long m, double &kx, double &ky, double &kz) {
  const int ix = (int)(m % g.nxh);
  const int iy = (int)((m / g.nxh) % g.ny);
  const int iz = (int)(m / ((long long)g.nxh * g.ny));
  kx = k_half(ix, g.nx, g.ax);
  ky = k_full(iy, g.ny, g.ay);
  kz = k_full(iz, g.nz, g.az);
}

// rhs.f90:74-88 mask (dealias, .ge., spherical factor 0.5, or k = 0)
__device__ __forceinline__ bool rhs_masked(const Grid3 &g, double kx, double ky, double kz) {
  const double k2 = kx * kx + ky * ky + kz * kz;
  return (g.spherical && k2 >= g.sph2) || fabs(kx) >= g.cutx || fabs(ky) >= g.cuty || fabs(kz) >= g.cutz ||
         (kx == 0.0 && ky == 0.0 && kz == 0.0);
}

// rhsAdj.f90:131-136 mask (.gt., no k = 0 term)
__device__ __forceinline__ bool adj_masked(const Grid3 &g, double kx, double ky, double kz) {
  return fabs(kx) > g.cutx || fabs(ky) > g.cuty || fabs(kz) > g.cutz;
}

#define GRID_LOOP(m, n)                                                                   \
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < (n);           \
       m += (long long)gridDim.x * blockDim.x)

// h / W = -P(D g) / W
template <typename C>
__global__ void k_vjp_pre(const C *g, C *hw, long long nh, Grid3 gr) {
  using T = decltype(C{}.x);
  GRID_LOOP(m, nh) {
    double kx, ky, kz;
    mode_k(gr, m, kx, ky, kz);
    if (rhs_masked(gr, kx, ky, kz)) {
      for (int c = 0; c < 3; ++c) hw[c * nh + m] = mkc<C>(0, 0);
      continue;
    }
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double kr[3] = {kx, ky, kz};
    const C v[3] = {g[m], g[nh + m], g[2 * nh + m]};
    const double dre = (kx * v[0].x + ky * v[1].x + kz * v[2].x) / k2;
    const double dim = (kx * v[0].y + ky * v[1].y + kz * v[2].y) / k2;
    const double w = (kx == 0.0) ? 1.0 : 0.5;   // 1 / W
    for (int c = 0; c < 3; ++c)
      hw[c * nh + m] = mkc<C>(T(-(v[c].x - kr[c] * dre) * w), T(-(v[c].y - kr[c] * dim) * w));
  }
}

// physical: u <- u x phi, omega <- phi x omega (u: f[0..2], omega: f[3..5], phi: f[6..8])
template <typename T>
__global__ void k_vjp_cross(T *f, long long np) {
  GRID_LOOP(i, np) {
    const T u0 = f[i], u1 = f[np + i], u2 = f[2 * np + i];
    const T o0 = f[3 * np + i], o1 = f[4 * np + i], o2 = f[5 * np + i];
    const T p0 = f[6 * np + i], p1 = f[7 * np + i], p2 = f[8 * np + i];
    f[i] = u1 * p2 - u2 * p1;
    f[np + i] = u2 * p0 - u0 * p2;
    f[2 * np + i] = u0 * p1 - u1 * p0;
    f[3 * np + i] = p1 * o2 - p2 * o1;
    f[4 * np + i] = p2 * o0 - p0 * o2;
    f[5 * np + i] = p0 * o1 - p1 * o0;
  }
}

// out = s W (ik x A + B)
template <typename C>
__global__ void k_vjp_combine(const C *A, const C *Bv, C *out, long long nh, Grid3 gr, double s) {
  using T = decltype(C{}.x);
  GRID_LOOP(m, nh) {
    double kx, ky, kz;
    mode_k(gr, m, kx, ky, kz);
    const double sw = s * ((kx == 0.0) ? 1.0 : 2.0);
    const C a0 = A[m], a1 = A[nh + m], a2 = A[2 * nh + m];
    // i (k x a): component = i (k_j a_k - k_k a_j)
    const double cx_re = -(ky * a2.y - kz * a1.y), cx_im = ky * a2.x - kz * a1.x;
    const double cy_re = -(kz * a0.y - kx * a2.y), cy_im = kz * a0.x - kx * a2.x;
    const double cz_re = -(kx * a1.y - ky * a0.y), cz_im = kx * a1.x - ky * a0.x;
    const C b0 = Bv[m], b1 = Bv[nh + m], b2 = Bv[2 * nh + m];
    out[m] = mkc<C>(T(sw * (cx_re + b0.x)), T(sw * (cx_im + b0.y)));
    out[nh + m] = mkc<C>(T(sw * (cy_re + b1.x)), T(sw * (cy_im + b1.y)));
    out[2 * nh + m] = mkc<C>(T(sw * (cz_re + b2.x)), T(sw * (cz_im + b2.y)));
  }
}

// Band forcing part of the VJP (one block): with c = Pin / (2 Eb),
// out += c (Bm g) - (Pin / (2 Eb^2)) <Bm u, g> 2 s^2 (w Bb u), where Bb are the
// band modes of rhs_Eband (weight w = 1/2 on kx = 0) and Bm those of them that
// the rhs.f90 mask keeps.
template <typename C>
__global__ void k_vjp_band(const C *u, const C *g, C *out, long long nh, const int *band, int nband, Grid3 gr,
                           const StepState *st, double Pin, double s2) {
  using T = decltype(C{}.x);
  __shared__ double red[32];
  const double eb = st->eband;
  double dot = 0.0;
  for (int i = threadIdx.x; i < nband; i += blockDim.x) {
    const long long off = (long long)(unsigned)band[3 * i] | ((long long)band[3 * i + 1] << 32);
    double kx, ky, kz;
    mode_k(gr, off, kx, ky, kz);
    if (rhs_masked(gr, kx, ky, kz)) continue;
    for (int c = 0; c < 3; ++c) {
      const C a = u[c * nh + off], b = g[c * nh + off];
      dot += (double)a.x * b.x + (double)a.y * b.y;
    }
  }
  double v[1] = {dot};
  block_sum<1>(v, red);
  __shared__ double dsh;
  if (threadIdx.x == 0) dsh = v[0];
  __syncthreads();
  dot = dsh;
  const double cf = Pin / (2.0 * eb), cg = Pin / (2.0 * eb * eb) * dot * 2.0 * s2;
  for (int i = threadIdx.x; i < nband; i += blockDim.x) {
    const long long off = (long long)(unsigned)band[3 * i] | ((long long)band[3 * i + 1] << 32);
    double kx, ky, kz;
    mode_k(gr, off, kx, ky, kz);
    const bool keep = !rhs_masked(gr, kx, ky, kz);
    const double w = (kx == 0.0) ? 0.5 : 1.0;
    for (int c = 0; c < 3; ++c) {
      const C a = u[c * nh + off], b = g[c * nh + off];
      C o = out[c * nh + off];
      double re = o.x - cg * w * a.x, im = o.y - cg * w * a.y;
      if (keep) {
        re += cf * b.x;
        im += cf * b.y;
      }
      out[c * nh + off] = mkc<C>(T(re), T(im));
    }
  }
}

// rhsAdj.f90:83-121: p_c = sum_j u_j d_j u_c * s  (u = f[0..2] unscaled, grad(c,j) = f[3+3c+j], out f[12..14])
template <typename T>
__global__ void k_conv_prod(T *f, long long np, double s) {
  GRID_LOOP(i, np) {
    const T u[3] = {f[i], f[np + i], f[2 * np + i]};
    for (int c = 0; c < 3; ++c) {
      T acc = 0;
      for (int j = 0; j < 3; ++j) acc += u[j] * f[(3 + 3 * c + j) * np + i];
      f[(12 + c) * np + i] = acc * T(s);
    }
  }
}

// rhsAdj.f90:271-309: q_c = (sum_j d_c r_j u_j + sum_j d_j r_c u_j) * s
template <typename T>
__global__ void k_adj_prod(T *f, long long np, double s) {
  GRID_LOOP(i, np) {
    const T u[3] = {f[i], f[np + i], f[2 * np + i]};
    for (int c = 0; c < 3; ++c) {
      T acc = 0;
      for (int j = 0; j < 3; ++j) acc += f[(3 + 3 * j + c) * np + i] * u[j] + f[(3 + 3 * c + j) * np + i] * u[j];
      f[(12 + c) * np + i] = acc * T(s);
    }
  }
}

// rhsAdj.f90 spectral loop (:128-169 / :311-352) on n -> N; stage 1 also forms
// r~ = H^-1 (L u + N) (rhsupptilde, :177-213); stage 2 forms rhsadj = L r~ + N_adj.
template <typename C>
__global__ void k_adj_finish(const C *n, const C *uin, C *out, long long nh, Grid3 gr, double nu, double Q,
                             int stage, int hminone, int phat_literal) {
  using T = decltype(C{}.x);
  GRID_LOOP(m, nh) {
    double kx, ky, kz;
    mode_k(gr, m, kx, ky, kz);
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double kr[3] = {kx, ky, kz};
    double N[3][2];
    if (adj_masked(gr, kx, ky, kz)) {
      for (int c = 0; c < 3; ++c) N[c][0] = N[c][1] = 0.0;
    } else {
      const double eps = (kx == 0.0 && ky == 0.0 && kz == 0.0) ? 1.0e-13 : 0.0;
      const C v[3] = {n[m], n[nh + m], n[2 * nh + m]};
      const double knre = kx * v[0].x + ky * v[1].x + kz * v[2].x;
      const double knim = kx * v[0].y + ky * v[1].y + kz * v[2].y;
      // phat = -(i k.n) / (-(k.k) + eps)
      double pre = knim / (-k2 + eps), pim = -knre / (-k2 + eps);
      if (stage == 2 && phat_literal) pre = pim = 0.0;   // phatadj never assigned (Q6)
      for (int c = 0; c < 3; ++c) {
        N[c][0] = -(double)v[c].x + kr[c] * pim;
        N[c][1] = -(double)v[c].y - kr[c] * pre;
      }
    }
    const double L = Q - nu * k2;
    if (stage == 1) {
      const double h = hminone ? 1.0 / (1.0 + k2) : 1.0;
      for (int c = 0; c < 3; ++c) {
        const C u = uin[c * nh + m];
        out[c * nh + m] = mkc<C>(T(h * (L * u.x + N[c][0])), T(h * (L * u.y + N[c][1])));
      }
    } else {
      for (int c = 0; c < 3; ++c) {
        const C r = uin[c * nh + m];
        out[c * nh + m] = mkc<C>(T(L * r.x + N[c][0]), T(L * r.y + N[c][1]));
      }
    }
  }
}

// r = L u + N (N already carries any fixed forcing); per-block partials of
// J = 1/2 s^2 sum W h |r|^2; gE = s^2 W h r
template <typename C>
__global__ void k_residual(const C *u, const C *N, C *gE, long long nh, Grid3 gr, double nu, double Q, int hminone,
                           double s2, double *partials) {
  using T = decltype(C{}.x);
  __shared__ double red[32];
  double acc = 0.0;
  GRID_LOOP(m, nh) {
    double kx, ky, kz;
    mode_k(gr, m, kx, ky, kz);
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double L = Q - nu * k2;
    const double h = hminone ? 1.0 / (1.0 + k2) : 1.0;
    const double W = (kx == 0.0) ? 1.0 : 2.0;
    for (int c = 0; c < 3; ++c) {
      const C a = u[c * nh + m], b = N[c * nh + m];
      const double re = L * a.x + b.x, im = L * a.y + b.y;
      acc += 0.5 * s2 * W * h * (re * re + im * im);
      if (gE) gE[c * nh + m] = mkc<C>(T(s2 * W * h * re), T(s2 * W * h * im));
    }
  }
  double v[1] = {acc};
  block_sum<1>(v, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

// grad += L gE
template <typename C>
__global__ void k_add_linear(C *grad, const C *gE, long long nh, Grid3 gr, double nu, double Q) {
  using T = decltype(C{}.x);
  GRID_LOOP(m, nh) {
    double kx, ky, kz;
    mode_k(gr, m, kx, ky, kz);
    const double L = Q - nu * (kx * kx + ky * ky + kz * kz);
    for (int c = 0; c < 3; ++c) {
      const C a = grad[c * nh + m], b = gE[c * nh + m];
      grad[c * nh + m] = mkc<C>(T(a.x + L * b.x), T(a.y + L * b.y));
    }
  }
}

// d = -P D (grad / (s^2 W)): the steepest-descent direction in the
// mean-square metric <|u|^2> = s^2 sum_half W |uhat|^2 of J's own norm,
// projected and dealiased so the state stays admissible; per-block partials
// of <grad, d>
template <typename C>
__global__ void k_descent_dir(const C *grad, C *d, long long nh, Grid3 gr, double s2, double *partials) {
  using T = decltype(C{}.x);
  __shared__ double red[32];
  double acc = 0.0;
  GRID_LOOP(m, nh) {
    double kx, ky, kz;
    mode_k(gr, m, kx, ky, kz);
    if (rhs_masked(gr, kx, ky, kz)) {
      for (int c = 0; c < 3; ++c) d[c * nh + m] = mkc<C>(0, 0);
      continue;
    }
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double kr[3] = {kx, ky, kz};
    const double w = ((kx == 0.0) ? 1.0 : 0.5) / s2;
    const C v[3] = {grad[m], grad[nh + m], grad[2 * nh + m]};
    const double dre = (kx * v[0].x + ky * v[1].x + kz * v[2].x) / k2;
    const double dim = (kx * v[0].y + ky * v[1].y + kz * v[2].y) / k2;
    for (int c = 0; c < 3; ++c) {
      const double re = -(v[c].x - kr[c] * dre) * w, im = -(v[c].y - kr[c] * dim) * w;
      d[c * nh + m] = mkc<C>(T(re), T(im));
      acc += re * v[c].x + im * v[c].y;
    }
  }
  double v[1] = {acc};
  block_sum<1>(v, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

// out = IF (u + dt n), IF = exp((Q - nu |k|^2) dt): the FIN_PRED arithmetic of k_finish_rows
template <typename C>
__global__ void k_if_pred(const C *u, const C *n, C *out, long long nh, Grid3 gr, double nu, double Q, double dt) {
  using T = decltype(C{}.x);
  GRID_LOOP(m, nh) {
    double kx, ky, kz;
    mode_k(gr, m, kx, ky, kz);
    const T IF = T(exp((Q - nu * (kx * kx + ky * ky + kz * kz)) * dt));
    const T tdt = T(dt);
    for (int c = 0; c < 3; ++c) {
      const C a = u[c * nh + m], b = n[c * nh + m];
      out[c * nh + m] = mkc<C>((a.x + tdt * b.x) * IF, (a.y + tdt * b.y) * IF);
    }
  }
}

// y = s x over n complex values
template <typename C>
__global__ void k_scale(const C *x, C *y, long long n, double s) {
  using T = decltype(C{}.x);
  GRID_LOOP(i, n) {
    const C a = x[i];
    y[i] = mkc<C>(T(s * a.x), T(s * a.y));
  }
}

// partial = IF (g + a), arg = IF (dt/2 g + dt a)
template <typename C>
__global__ void k_step_mix(const C *g, const C *a, C *partial, C *arg, long long nh, Grid3 gr, double nu, double Q,
                           double dt) {
  using T = decltype(C{}.x);
  GRID_LOOP(m, nh) {
    double kx, ky, kz;
    mode_k(gr, m, kx, ky, kz);
    const double IF = exp((Q - nu * (kx * kx + ky * ky + kz * kz)) * dt);
    for (int c = 0; c < 3; ++c) {
      const C gg = g[c * nh + m], aa = a[c * nh + m];
      partial[c * nh + m] = mkc<C>(T(IF * ((double)gg.x + aa.x)), T(IF * ((double)gg.y + aa.y)));
      arg[c * nh + m] = mkc<C>(T(IF * (0.5 * dt * gg.x + dt * aa.x)), T(IF * (0.5 * dt * gg.y + dt * aa.y)));
    }
  }
}

// y += x over n complex values
template <typename C>
__global__ void k_accum(C *y, const C *x, long long n, double sx) {
  using T = decltype(C{}.x);
  GRID_LOOP(i, n) {
    const C a = y[i], b = x[i];
    y[i] = mkc<C>(T(a.x + sx * b.x), T(a.y + sx * b.y));
  }
}

// r = uT - u0, g = s^2 W r, per-block partial sums of 1/2 s^2 W |r|^2
template <typename C>
__global__ void k_orbit_res(const C *uT, const C *u0, C *g, long long nh, Grid3 gr, double s2, double *partials) {
  using T = decltype(C{}.x);
  __shared__ double red[32];
  double acc = 0.0;
  GRID_LOOP(m, nh) {
    double kx, ky, kz;
    mode_k(gr, m, kx, ky, kz);
    const double w = (kx == 0.0) ? 1.0 : 2.0;   // half-spectrum multiplicity (kx = 0 and Nyquist planes: 1)
    for (int c = 0; c < 3; ++c) {
      const C a = uT[c * nh + m], b = u0[c * nh + m];
      const double re = (double)a.x - b.x, im = (double)a.y - b.y;
      acc += 0.5 * s2 * w * (re * re + im * im);
      g[c * nh + m] = mkc<C>(T(s2 * w * re), T(s2 * w * im));
    }
  }
  double v[1] = {acc};
  block_sum<1>(v, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

constexpr int kRedBlocks = 148 * 2;

Grid3 grid3(const dnsbox_ctx *c) {
  const dnsbox_params &p = c->p;
  Grid3 g;
  g.nx = p.nx;
  g.ny = p.ny;
  g.nz = p.nz;
  g.nxh = c->nxh;
  g.ax = p.alpha_x;
  g.ay = p.alpha_y;
  g.az = p.alpha_z;
  g.cutx = (p.nx / 2.0) * (2.0 * p.alpha_x / 3.0);
  g.cuty = (p.ny / 2.0) * (2.0 * p.alpha_y / 3.0);
  g.cutz = (p.nz / 2.0) * (2.0 * p.alpha_z / 3.0);
  g.sph2 = pow((p.nx / 2.0) * 0.5 * p.alpha_x, 2);
  g.spherical = p.spherical;
  return g;
}

// adjoint arena: nphys physical fields followed by nspec spectral fields
int ensure_adj(dnsbox_ctx *c, int nphys, int nspec, char **phys, char **spec) {
  const size_t pb = c->np * (c->cbytes / 2), sb = c->nh * c->cbytes;
  const size_t need = nphys * pb + nspec * sb;
  if (need > c->adj_bytes) {
    if (c->adj) cudaFree(c->adj);
    c->adj = nullptr;
    c->adj_bytes = 0;
    CK(cudaMalloc(&c->adj, need));
    c->adj_bytes = need;
  }
  *phys = c->adj;
  *spec = c->adj + nphys * pb;
  return DNSBOX_OK;
}

int sum_to_host(dnsbox_ctx *c, int nblk, double *out) {
  k_sum_scalar<256><<<1, 256, 0, c->stream>>>(c->red, nblk, c->red + nblk);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->hstage, c->red + nblk, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  RET(tc_check(c));
  *out = c->hstage[0];
  return DNSBOX_OK;
}

template <typename T>
int vjp_impl(dnsbox_ctx *c, const void *uh, const void *g, void *out) {
  using C = typename CT<T>::type;
  const dnsbox_params &p = c->p;
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  const size_t pb = c->np * sizeof(T), sb = c->nh * sizeof(C);
  char *P = nullptr, *S = nullptr;
  RET(ensure_adj(c, 9, 6, &P, &S));
  const Grid3 gr = grid3(c);
  const int gb = grid_for((long long)c->nh);
  const long long nh = (long long)c->nh, np = (long long)c->np;
  const char *u = reinterpret_cast<const char *>(uh);
  k_vjp_pre<C><<<gb, 256, 0, c->stream>>>(reinterpret_cast<const C *>(g), reinterpret_cast<C *>(S), nh, gr);
  CK(cudaGetLastError());
  // u (scaled), omega = ik x u (scaled), phi = C2R(h / W)
  const void *u0 = u, *u1 = u + sb, *u2 = u + 2 * sb;
  SpecJob jobs[9] = {
      {{{u0, s, 0, 0}, {nullptr, 0, 0, 0}}, 1},
      {{{u1, s, 0, 0}, {nullptr, 0, 0, 0}}, 1},
      {{{u2, s, 0, 0}, {nullptr, 0, 0, 0}}, 1},
      {{{u2, 0, s, 2}, {u1, 0, -s, 1}}, 2},   // i (ky w - kz v)
      {{{u0, 0, s, 1}, {u2, 0, -s, 0}}, 2},   // i (kz u - kx w)
      {{{u1, 0, s, 0}, {u0, 0, -s, 2}}, 2},   // i (kx v - ky u)
      {{{S, 1, 0, 0}, {nullptr, 0, 0, 0}}, 1},
      {{{S + sb, 1, 0, 0}, {nullptr, 0, 0, 0}}, 1},
      {{{S + 2 * sb, 1, 0, 0}, {nullptr, 0, 0, 0}}, 1},
  };
  void *outs[9];
  for (int i = 0; i < 9; ++i) outs[i] = P + i * pb;
  RET(c2r_jobs<T>(c, 9, jobs, outs, 1.0));
  k_vjp_cross<T><<<grid_for(np), 256, 0, c->stream>>>(reinterpret_cast<T *>(P), np);
  CK(cudaGetLastError());
  const void *ins[6];
  void *specs[6];
  for (int i = 0; i < 6; ++i) {
    ins[i] = P + i * pb;
    specs[i] = S + i * sb;
  }
  RET(r2c_fields<T>(c, 6, ins, specs));
  k_vjp_combine<C><<<gb, 256, 0, c->stream>>>(reinterpret_cast<const C *>(S), reinterpret_cast<const C *>(S + 3 * sb),
                                              reinterpret_cast<C *>(out), nh, gr, s);
  CK(cudaGetLastError());
  if (p.bandlim && c->nband) {
    k_eband<C><<<1, 256, 0, c->stream>>>(reinterpret_cast<const C *>(uh), nh, c->band, c->nband, p.nx, c->st,
                                         s * s, 0);
    k_vjp_band<C><<<1, 256, 0, c->stream>>>(reinterpret_cast<const C *>(uh), reinterpret_cast<const C *>(g),
                                            reinterpret_cast<C *>(out), nh, c->band, c->nband, gr, c->st, p.Pin,
                                            s * s);
    CK(cudaGetLastError());
  }
  return DNSBOX_OK;
}

template <typename T>
int rhs_adj_impl(dnsbox_ctx *c, const void *uh, void *rt, void *rhsadj) {
  using C = typename CT<T>::type;
  const dnsbox_params &p = c->p;
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  const size_t pb = c->np * sizeof(T), sb = c->nh * sizeof(C);
  char *P = nullptr, *S = nullptr;
  RET(ensure_adj(c, 15, 3, &P, &S));
  const Grid3 gr = grid3(c);
  const int gb = grid_for((long long)c->nh);
  const long long nh = (long long)c->nh, np = (long long)c->np;
  const char *u = reinterpret_cast<const char *>(uh);
  const int ks_of_dir[3] = {0, 2, 1};   // d/dx: kx, d/dy: ky (other axis of the z pass), d/dz: kz (row)
  // stage 1: u (unscaled, x N^3) and grad u (rhsAdj.f90:8-52, 75-77)
  SpecJob jobs[12];
  for (int cc = 0; cc < 3; ++cc) jobs[cc] = SpecJob{{{u + cc * sb, 1.0, 0.0, 0}, {nullptr, 0, 0, 0}}, 1};
  for (int cc = 0; cc < 3; ++cc)
    for (int j = 0; j < 3; ++j)
      jobs[3 + 3 * cc + j] = SpecJob{{{u + cc * sb, 0.0, s, ks_of_dir[j]}, {nullptr, 0, 0, 0}}, 1};
  void *outs[12];
  for (int i = 0; i < 12; ++i) outs[i] = P + i * pb;
  RET(c2r_jobs<T>(c, 12, jobs, outs, 1.0));
  k_conv_prod<T><<<grid_for(np), 256, 0, c->stream>>>(reinterpret_cast<T *>(P), np, s);
  CK(cudaGetLastError());
  const void *ins[3] = {P + 12 * pb, P + 13 * pb, P + 14 * pb};
  void *specs[3] = {S, S + sb, S + 2 * sb};
  RET(r2c_fields<T>(c, 3, ins, specs));
  k_adj_finish<C><<<gb, 256, 0, c->stream>>>(reinterpret_cast<const C *>(S), reinterpret_cast<const C *>(uh),
                                             reinterpret_cast<C *>(rt), nh, gr, p.nu, p.Q, 1, p.hminone, 0);
  CK(cudaGetLastError());
  // stage 2: grad r~ (rhsAdj.f90:215-259), products, adjoint term
  const char *r = reinterpret_cast<const char *>(rt);
  SpecJob jobs2[9];
  for (int cc = 0; cc < 3; ++cc)
    for (int j = 0; j < 3; ++j)
      jobs2[3 * cc + j] = SpecJob{{{r + cc * sb, 0.0, s, ks_of_dir[j]}, {nullptr, 0, 0, 0}}, 1};
  RET(c2r_jobs<T>(c, 9, jobs2, outs + 3, 1.0));
  k_adj_prod<T><<<grid_for(np), 256, 0, c->stream>>>(reinterpret_cast<T *>(P), np, s);
  CK(cudaGetLastError());
  RET(r2c_fields<T>(c, 3, ins, specs));
  k_adj_finish<C><<<gb, 256, 0, c->stream>>>(reinterpret_cast<const C *>(S), reinterpret_cast<const C *>(rt),
                                             reinterpret_cast<C *>(rhsadj), nh, gr, p.nu, p.Q, 2, p.hminone,
                                             p.adj_phat == DNSBOX_ADJ_PHAT_LITERAL);
  CK(cudaGetLastError());
  return DNSBOX_OK;
}

// Forward half of the residual: N(u) and the per-block partials of J into
// `partials` (kRedBlocks doubles), and, when `weighted` is set, the weighted
// residual that the gradient half transposes (arena slots 6-11).  No
// synchronisation.
template <typename T>
int residual_fwd(dnsbox_ctx *c, const void *uh, bool weighted, double *partials) {
  using C = typename CT<T>::type;
  const dnsbox_params &p = c->p;
  const double s = 1.0 / ((double)p.nx * p.ny * p.nz);
  const size_t sb = c->nh * sizeof(C);
  char *P = nullptr, *S = nullptr;
  RET(ensure_adj(c, 9, 12, &P, &S));
  char *Nb = S + 6 * sb, *gE = S + 9 * sb;
  RET(rhs_nonlinear_impl(c, uh, Nb));
  const Grid3 gr = grid3(c);
  k_residual<C><<<kRedBlocks, 256, 0, c->stream>>>(
      reinterpret_cast<const C *>(uh), reinterpret_cast<const C *>(Nb), weighted ? reinterpret_cast<C *>(gE) : nullptr,
      (long long)c->nh, gr, p.nu, p.Q, p.hminone, s * s, partials);
  CK(cudaGetLastError());
  return DNSBOX_OK;
}

// Gradient half: grad = (L + N'(u))^T applied to the weighted residual that
// the last residual_fwd(uh, weighted) left in the arena.
template <typename T>
int residual_bwd(dnsbox_ctx *c, const void *uh, void *grad) {
  using C = typename CT<T>::type;
  const dnsbox_params &p = c->p;
  const size_t sb = c->nh * sizeof(C);
  char *P = nullptr, *S = nullptr;
  RET(ensure_adj(c, 9, 12, &P, &S));
  char *gE = S + 9 * sb;
  const Grid3 gr = grid3(c);
  RET(vjp_impl<T>(c, uh, gE, grad));
  k_add_linear<C><<<grid_for((long long)c->nh), 256, 0, c->stream>>>(
      reinterpret_cast<C *>(grad), reinterpret_cast<const C *>(gE), (long long)c->nh, gr, p.nu, p.Q);
  CK(cudaGetLastError());
  return DNSBOX_OK;
}

// J (and, when grad != null, its Euclidean gradient) at uh.  Uses arena
// spectral slots 6-8 for N and 9-11 for gE (slots 0-5 belong to the VJP).
template <typename T>
int residual_impl(dnsbox_ctx *c, const void *uh, void *grad, double *J) {
  RET(ensure_red(c, 2 * kRedBlocks + 2));
  RET(residual_fwd<T>(c, uh, grad != nullptr, c->red));
  RET(sum_to_host(c, kRedBlocks, J));
  if (grad) RET(residual_bwd<T>(c, uh, grad));
  return DNSBOX_OK;
}

// y = x + alpha d with alpha read from device memory (the launch is part of a
// captured graph whose step length changes between launches)
template <typename C>
__global__ void k_axpy_dev(const C *x, const C *d, C *y, long long n, const double *alpha_p) {
  using T = decltype(C{}.x);
  const double alpha = *alpha_p;
  GRID_LOOP(i, n) {
    const C a = x[i], b = d[i];
    y[i] = mkc<C>(T(a.x + alpha * b.x), T(a.y + alpha * b.y));
  }
}

}  // namespace

// The adjoint descent's fixed launch sequences as CUDA graphs, on a private
// stream: the descent direction with the slope sum; per buffer parity p (state
// in buffer p, trial in buffer 1 - p) the trial (axpy with the device step
// length, forward residual, J sum, read-back of slope and J into pinned host
// memory) and the gradient half at the trial.  Valid while the state pointer
// and the scratch buffers they were captured with are unchanged.
struct DescentGraphs {
  cudaStream_t s = nullptr;
  cudaEvent_t ev = nullptr;
  cudaGraphExec_t dir = nullptr, tryg[2] = {nullptr, nullptr}, bwd[2] = {nullptr, nullptr};
  const void *uh = nullptr;
  const char *adj = nullptr;
  const double *red = nullptr;
  const void *force = nullptr;   // the fixed forcing the captured finish launches read
  int fp64 = -1;
};

static void graphs_destroy(DescentGraphs *g) {
  if (!g) return;
  if (g->dir) cudaGraphExecDestroy(g->dir);
  for (int i = 0; i < 2; ++i) {
    if (g->tryg[i]) cudaGraphExecDestroy(g->tryg[i]);
    if (g->bwd[i]) cudaGraphExecDestroy(g->bwd[i]);
  }
  if (g->ev) cudaEventDestroy(g->ev);
  if (g->s) cudaStreamDestroy(g->s);
  delete g;
}

void descent_graphs_free(dnsbox_ctx *c) {
  graphs_destroy(c->descent);
  c->descent = nullptr;
}

namespace {

// Captures the launches f() makes on the context's stream (redirected to s)
// into an executable graph.  Pass-event profiling is off during the capture.
template <typename F>
static int capture_graph(dnsbox_ctx *c, cudaStream_t s, F &&f, cudaGraphExec_t *out) {
  cudaStream_t saved = c->stream;
  const int prof = c->prof_on;
  c->stream = s;
  c->prof_on = 0;
  const cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  const int rc = e == cudaSuccess ? f() : DNSBOX_OK;
  cudaGraph_t graph = nullptr;
  const cudaError_t e2 = e == cudaSuccess ? cudaStreamEndCapture(s, &graph) : e;
  c->stream = saved;
  c->prof_on = prof;
  if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "cudaStreamBeginCapture: %s", cudaGetErrorString(e));
  if (rc != DNSBOX_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e2 != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e2));
  const cudaError_t e3 = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e3 != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e3));
  return DNSBOX_OK;
}

// Steepest descent on J with an FP64 Armijo line search.  The state alternates
// between uh and the trial slot: an accepted trial's forward half (J and the
// weighted residual) is kept, so only the gradient half runs at the new
// point, and the slope <grad, d> is read back together with the first trial's
// J (one synchronisation per trial).  After the first residual (which grows
// every scratch buffer) the iterations run as graph launches.
template <typename T>
int descent_impl(dnsbox_ctx *c, void *uh, int niter, double *Jhist, double *alpha_io) {
  using C = typename CT<T>::type;
  const size_t sb = c->nh * sizeof(C);
  char *P = nullptr, *S = nullptr;
  RET(ensure_adj(c, 9, 21, &P, &S));
  char *grad = S + 12 * sb, *dir = S + 15 * sb, *trial = S + 18 * sb;
  const Grid3 gr = grid3(c);
  const long long n3 = 3 * (long long)c->nh;
  double alpha = (alpha_io && *alpha_io > 0) ? *alpha_io : 1.0;
  double J = 0.0;
  RET(ensure_red(c, 2 * kRedBlocks + 4));
  RET(residual_impl<T>(c, uh, grad, &J));
  if (Jhist) Jhist[0] = J;
  if (niter <= 0) {
    if (alpha_io) *alpha_io = alpha;
    return DNSBOX_OK;
  }
  double *red = c->red, *d_alpha = c->red + 2 * kRedBlocks + 2;
  double *h_alpha = c->hstage + 40, *h_res = c->hstage + 41;   // pinned: step length out, (slope, J) in
  const double s = 1.0 / ((double)c->p.nx * c->p.ny * c->p.nz), s2 = s * s;
  char *buf[2] = {reinterpret_cast<char *>(uh), trial};
  DescentGraphs *g = c->descent;
  if (g && (g->uh != uh || g->adj != c->adj || g->red != c->red || g->fp64 != c->fp64 || g->force != c->force)) {
    descent_graphs_free(c);
    g = nullptr;
  }
  if (!g) {
    // built aside and kept only when every capture succeeded
    std::unique_ptr<DescentGraphs, void (*)(DescentGraphs *)> ng(new DescentGraphs(), graphs_destroy);
    g = ng.get();
    g->uh = uh;
    g->adj = c->adj;
    g->red = c->red;
    g->force = c->force;
    g->fp64 = c->fp64;
    CK(cudaStreamCreateWithFlags(&g->s, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&g->ev, cudaEventDisableTiming));
    RET(capture_graph(c, g->s, [&]() -> int {
      k_descent_dir<C><<<kRedBlocks, 256, 0, c->stream>>>(reinterpret_cast<const C *>(grad), reinterpret_cast<C *>(dir),
                                                          (long long)c->nh, gr, s2, red);
      k_sum_scalar<256><<<1, 256, 0, c->stream>>>(red, kRedBlocks, red + 2 * kRedBlocks);
      CK(cudaGetLastError());
      return DNSBOX_OK;
    }, &g->dir));
    for (int p = 0; p < 2; ++p) {
      char *cur = buf[p], *nxt = buf[1 - p];
      RET(capture_graph(c, g->s, [&]() -> int {
        k_axpy_dev<C><<<grid_for(n3), 256, 0, c->stream>>>(reinterpret_cast<const C *>(cur),
                                                           reinterpret_cast<const C *>(dir), reinterpret_cast<C *>(nxt),
                                                           n3, d_alpha);
        CK(cudaGetLastError());
        RET(residual_fwd<T>(c, nxt, true, red + kRedBlocks));
        k_sum_scalar<256><<<1, 256, 0, c->stream>>>(red + kRedBlocks, kRedBlocks, red + 2 * kRedBlocks + 1);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(h_res, red + 2 * kRedBlocks, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        return DNSBOX_OK;
      }, &g->tryg[p]));
      RET(capture_graph(c, g->s, [&]() -> int { return residual_bwd<T>(c, nxt, grad); }, &g->bwd[p]));
    }
    c->descent = ng.release();
  }
  // the graphs run on g->s after the work queued so far on the context's stream
  CK(cudaEventRecord(g->ev, c->stream));
  CK(cudaStreamWaitEvent(g->s, g->ev, 0));
  int p = 0;   // the state is in buf[p]
  for (int it = 0; it < niter; ++it) {
    CK(cudaGraphLaunch(g->dir, g->s));
    // Armijo backtracking in FP64: J(u + a d) <= J + 1e-4 a <grad, d>
    double slope = 0.0, Jt = 0.0;
    int tries = 0;
    bool stationary = false;
    for (;;) {
      *h_alpha = alpha;   // the previous copy of this slot has completed (synchronised below)
      CK(cudaMemcpyAsync(d_alpha, h_alpha, sizeof(double), cudaMemcpyHostToDevice, g->s));
      CK(cudaGraphLaunch(g->tryg[p], g->s));
      CK(cudaStreamSynchronize(g->s));
      slope = h_res[0];
      Jt = h_res[1];
      if (!(slope < 0.0)) {   // stationary (or non-finite)
        stationary = true;
        break;
      }
      if ((isfinite(Jt) && Jt <= J + 1e-4 * alpha * slope) || ++tries >= 30) break;
      alpha *= 0.5;
    }
    if (stationary || !(isfinite(Jt) && Jt <= J)) break;
    CK(cudaGraphLaunch(g->bwd[p], g->s));
    p ^= 1;   // the accepted trial becomes the state; the old state's buffer the next trial
    J = Jt;
    if (Jhist) Jhist[it + 1] = J;
    if (tries == 0) alpha *= 2.0;
  }
  if (p) CK(cudaMemcpyAsync(uh, buf[1], 3 * sb, cudaMemcpyDeviceToDevice, g->s));
  CK(cudaEventRecord(g->ev, g->s));
  CK(cudaStreamWaitEvent(c->stream, g->ev, 0));
  if (alpha_io) *alpha_io = alpha;
  RET(tc_check(c));
  return DNSBOX_OK;
}

// The adjoint arena and the residual reductions hold one box: batched
// contexts are refused before anything is launched.
static int single_box(dnsbox_ctx *c) {
  if (c->nbatch > 1)
    return set_err(DNSBOX_ERR_UNSUPPORTED, "not available on a batched context (nbatch = %d)", c->nbatch);
  return DNSBOX_OK;
}

// Checks that a context can be differentiated step by step: one box, IF-Heun,
// fixed dt (the CFL rule makes dt depend on max |u_i|, which has no useful
// derivative).
int step_vjp_ok(dnsbox_ctx *c) {
  if (c->nbatch > 1) return set_err(DNSBOX_ERR_UNSUPPORTED, "not available on a batched context");
  if (c->p.stepper != DNSBOX_HEUN) return set_err(DNSBOX_ERR_UNSUPPORTED, "step transpose needs the Heun stepper");
  if (!c->p.tstep_fix) return set_err(DNSBOX_ERR_UNSUPPORTED, "step transpose needs a fixed time step (tstep_fix)");
  return DNSBOX_OK;
}

// One step transpose: out = S'(u)^T g.  Arena spectral slots 21-32 (0-5 belong
// to the rhs VJP).  out may not alias u or g.
template <typename T>
int step_vjp_impl(dnsbox_ctx *c, const void *uh, const void *g, void *out, double dt) {
  using C = typename CT<T>::type;
  const dnsbox_params &p = c->p;
  const size_t sb = c->nh * sizeof(C);
  char *P = nullptr, *S = nullptr;
  RET(ensure_adj(c, 9, 33, &P, &S));
  char *n0 = S + 21 * sb, *ust = S + 24 * sb, *A = S + 27 * sb, *tmp = S + 30 * sb;
  const Grid3 gr = grid3(c);
  const long long nh = (long long)c->nh, n3 = 3 * nh;
  {
    const int rc = dnsbox_rhs_nonlinear(c, uh, n0, nullptr);
    if (rc != DNSBOX_OK) return rc;
  }
  k_if_pred<C><<<grid_for(nh), 256, 0, c->stream>>>(reinterpret_cast<const C *>(uh), reinterpret_cast<const C *>(n0),
                                                     reinterpret_cast<C *>(ust), nh, gr, p.nu, p.Q, dt);
  k_scale<C><<<grid_for(n3), 256, 0, c->stream>>>(reinterpret_cast<const C *>(g), reinterpret_cast<C *>(tmp), n3,
                                                   0.5 * dt);
  CK(cudaGetLastError());
  RET(vjp_impl<T>(c, ust, tmp, A));                       // a = N'(u*)^T (dt/2 g)
  k_step_mix<C><<<grid_for(nh), 256, 0, c->stream>>>(reinterpret_cast<const C *>(g), reinterpret_cast<const C *>(A),
                                                      reinterpret_cast<C *>(out), reinterpret_cast<C *>(tmp), nh, gr,
                                                      p.nu, p.Q, dt);
  CK(cudaGetLastError());
  RET(vjp_impl<T>(c, uh, tmp, n0));                       // N'(u)^T (IF (dt/2 g + dt a))
  k_accum<C><<<grid_for(n3), 256, 0, c->stream>>>(reinterpret_cast<C *>(out), reinterpret_cast<const C *>(n0), n3,
                                                   1.0);
  CK(cudaGetLastError());
  return DNSBOX_OK;
}

int ensure_orbit(dnsbox_ctx *c, size_t bytes) {
  if (bytes <= c->orbit_bytes) return DNSBOX_OK;
  if (c->orbit) cudaFree(c->orbit);
  c->orbit = nullptr;
  c->orbit_bytes = 0;
  CK(cudaMalloc(&c->orbit, bytes));
  c->orbit_bytes = bytes;
  return DNSBOX_OK;
}

// g0 = (Phi^nsteps)'(u0)^T gT, checkpoints every `every` steps.  Also leaves
// u(T) in *uT_out when non-null.  States advance with dnsbox_step, the
// library's fused step.
template <typename T>
int steps_vjp_impl(dnsbox_ctx *c, const void *u0, int nsteps, int every, const void *gT, void *g0, void *uT_out) {
  using C = typename CT<T>::type;
  const size_t sb3 = 3 * c->nh * sizeof(C);
  const int ncp = (nsteps + every - 1) / every;
  RET(ensure_orbit(c, (size_t)(ncp + every + 2) * sb3));
  char *cp = c->orbit, *seg = cp + (size_t)ncp * sb3, *ga = seg + (size_t)every * sb3, *gb = ga + sb3;
  double dt = 0.0;
  RET(dnsbox_get_dt(c, &dt));
  // forward sweep: checkpoints
  CK(cudaMemcpyAsync(seg, u0, sb3, cudaMemcpyDeviceToDevice, c->stream));
  for (int n = 0; n < nsteps; ++n) {
    if (n % every == 0) CK(cudaMemcpyAsync(cp + (size_t)(n / every) * sb3, seg, sb3, cudaMemcpyDeviceToDevice, c->stream));
    RET(step_advance_decided(c, seg, 1, n == 0));   // pruning decided once for the trajectory
  }
  if (uT_out) CK(cudaMemcpyAsync(uT_out, seg, sb3, cudaMemcpyDeviceToDevice, c->stream));
  // backward sweep, one segment at a time
  CK(cudaMemcpyAsync(ga, gT, sb3, cudaMemcpyDeviceToDevice, c->stream));
  for (int k = ncp - 1; k >= 0; --k) {
    const int n0 = k * every, len = (nsteps - n0 < every) ? nsteps - n0 : every;
    CK(cudaMemcpyAsync(seg, cp + (size_t)k * sb3, sb3, cudaMemcpyDeviceToDevice, c->stream));
    for (int j = 1; j < len; ++j) {
      CK(cudaMemcpyAsync(seg + (size_t)j * sb3, seg + (size_t)(j - 1) * sb3, sb3, cudaMemcpyDeviceToDevice,
                         c->stream));
      RET(step_advance_decided(c, seg + (size_t)j * sb3, 1, false));
    }
    for (int j = len - 1; j >= 0; --j) {
      RET(step_vjp_impl<T>(c, seg + (size_t)j * sb3, ga, gb, dt));
      char *t = ga;
      ga = gb;
      gb = t;
    }
  }
  CK(cudaMemcpyAsync(g0, ga, sb3, cudaMemcpyDeviceToDevice, c->stream));
  RET(tc_check(c));
  return DNSBOX_OK;
}

// J = 1/2 s^2 sum_half W |u(T) - u0|^2 and, when grad != null, (Phi'^T - I)(s^2 W r).
template <typename T>
int orbit_impl(dnsbox_ctx *c, const void *u0, int nsteps, int every, void *grad, double *J) {
  using C = typename CT<T>::type;
  const size_t sb = c->nh * sizeof(C);
  char *P = nullptr, *S = nullptr;
  RET(ensure_adj(c, 9, 39, &P, &S));
  char *uT = S + 33 * sb, *gc = S + 36 * sb;
  const Grid3 gr = grid3(c);
  const long long nh = (long long)c->nh;
  const double s = 1.0 / ((double)c->p.nx * c->p.ny * c->p.nz);
  CK(cudaMemcpyAsync(uT, u0, 3 * sb, cudaMemcpyDeviceToDevice, c->stream));
  RET(dnsbox_step(c, uT, nsteps, nullptr));
  RET(ensure_red(c, kRedBlocks + 1));
  k_orbit_res<C><<<kRedBlocks, 256, 0, c->stream>>>(reinterpret_cast<const C *>(uT), reinterpret_cast<const C *>(u0),
                                                     reinterpret_cast<C *>(gc), nh, gr, s * s, c->red);
  CK(cudaGetLastError());
  RET(sum_to_host(c, kRedBlocks, J));
  if (grad) {
    RET(steps_vjp_impl<T>(c, u0, nsteps, every, gc, grad, nullptr));
    k_accum<C><<<grid_for(3 * nh), 256, 0, c->stream>>>(reinterpret_cast<C *>(grad), reinterpret_cast<const C *>(gc),
                                                         3 * nh, -1.0);
    CK(cudaGetLastError());
    RET(tc_check(c));
  }
  return DNSBOX_OK;
}

}  // namespace

extern "C" int dnsbox_heun_step_vjp(dnsbox_ctx *ctx, const void *uh, const void *g, void *out) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  CK(cudaSetDevice(ctx->p.device));
  if (!uh || !g || !out) return set_err(DNSBOX_ERR_ARG, "null pointer");
  if (out == uh || out == g) return set_err(DNSBOX_ERR_ARG, "output may not alias an input");
  RET(step_vjp_ok(ctx));
  double dt = 0.0;
  RET(dnsbox_get_dt(ctx, &dt));
  return ctx->fp64 ? step_vjp_impl<double>(ctx, uh, g, out, dt) : step_vjp_impl<float>(ctx, uh, g, out, dt);
}

extern "C" int dnsbox_heun_steps_vjp(dnsbox_ctx *ctx, const void *u0, int nsteps, int every, const void *gT,
                                     void *g0, void *uT) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  CK(cudaSetDevice(ctx->p.device));
  if (!u0 || !gT || !g0) return set_err(DNSBOX_ERR_ARG, "null pointer");
  if (nsteps < 1 || every < 1) return set_err(DNSBOX_ERR_ARG, "nsteps and every must be positive");
  RET(step_vjp_ok(ctx));
  return ctx->fp64 ? steps_vjp_impl<double>(ctx, u0, nsteps, every, gT, g0, uT)
                   : steps_vjp_impl<float>(ctx, u0, nsteps, every, gT, g0, uT);
}

extern "C" int dnsbox_orbit_residual(dnsbox_ctx *ctx, const void *u0, int nsteps, int every, void *grad,
                                     double *J) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  CK(cudaSetDevice(ctx->p.device));
  if (!u0 || !J) return set_err(DNSBOX_ERR_ARG, "null pointer");
  if (nsteps < 1 || every < 1) return set_err(DNSBOX_ERR_ARG, "nsteps and every must be positive");
  if (grad == u0) return set_err(DNSBOX_ERR_ARG, "output may not alias the input");
  RET(step_vjp_ok(ctx));
  return ctx->fp64 ? orbit_impl<double>(ctx, u0, nsteps, every, grad, J)
                   : orbit_impl<float>(ctx, u0, nsteps, every, grad, J);
}

extern "C" int dnsbox_rhs_nonlinear_vjp(dnsbox_ctx *ctx, const void *uh, const void *g, void *out) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  RET(single_box(ctx));
  CK(cudaSetDevice(ctx->p.device));
  if (!uh || !g || !out) return set_err(DNSBOX_ERR_ARG, "null pointer");
  if (out == uh || out == g) return set_err(DNSBOX_ERR_ARG, "output may not alias an input");
  return ctx->fp64 ? vjp_impl<double>(ctx, uh, g, out) : vjp_impl<float>(ctx, uh, g, out);
}

extern "C" int dnsbox_rhs_adj(dnsbox_ctx *ctx, const void *uh, void *rt, void *rhsadj) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  RET(single_box(ctx));
  CK(cudaSetDevice(ctx->p.device));
  if (!uh || !rt || !rhsadj) return set_err(DNSBOX_ERR_ARG, "null pointer");
  if (rt == uh || rhsadj == uh || rt == rhsadj) return set_err(DNSBOX_ERR_ARG, "outputs may not alias");
  return ctx->fp64 ? rhs_adj_impl<double>(ctx, uh, rt, rhsadj) : rhs_adj_impl<float>(ctx, uh, rt, rhsadj);
}

extern "C" int dnsbox_residual(dnsbox_ctx *ctx, const void *uh, double *J) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  RET(single_box(ctx));
  CK(cudaSetDevice(ctx->p.device));
  if (!uh || !J) return set_err(DNSBOX_ERR_ARG, "null pointer");
  return ctx->fp64 ? residual_impl<double>(ctx, uh, nullptr, J) : residual_impl<float>(ctx, uh, nullptr, J);
}

extern "C" int dnsbox_residual_grad(dnsbox_ctx *ctx, const void *uh, void *grad, double *J) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  RET(single_box(ctx));
  CK(cudaSetDevice(ctx->p.device));
  if (!uh || !grad || !J) return set_err(DNSBOX_ERR_ARG, "null pointer");
  if (grad == uh) return set_err(DNSBOX_ERR_ARG, "output may not alias the input");
  return ctx->fp64 ? residual_impl<double>(ctx, uh, grad, J) : residual_impl<float>(ctx, uh, grad, J);
}

extern "C" int dnsbox_adjoint_descent(dnsbox_ctx *ctx, void *uh, int niter, double *Jhist, double *alpha) {
  if (!ctx) return set_err(DNSBOX_ERR_ARG, "null context");
  RET(single_box(ctx));
  CK(cudaSetDevice(ctx->p.device));
  if (!uh || niter < 0) return set_err(DNSBOX_ERR_ARG, "invalid argument");
  return ctx->fp64 ? descent_impl<double>(ctx, uh, niter, Jhist, alpha)
                   : descent_impl<float>(ctx, uh, niter, Jhist, alpha);
}
