// Internal host-side definitions shared by the translation units of
// libdnsbox_gpu.so: the context, error reporting, launch accounting and the
// transform helpers built on the pass kernels.
#pragma once

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/dnsbox.h"
#include "launch.cuh"

using namespace dnsbox;

// ------------------------------------------------------------------ errors
// Records the message returned by dnsbox_last_error() and returns `code`.
int set_err(int code, const char *fmt, ...);

#define CK(call)                                                                           \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return set_err(e_ == cudaErrorMemoryAllocation ? DNSBOX_ERR_OOM : DNSBOX_ERR_CUDA,  \
                     "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));   \
  } while (0)

#define RET(call)                     \
  do {                                \
    int r_ = (call);                  \
    if (r_ != DNSBOX_OK) return r_;   \
  } while (0)

struct dnsbox_ctx;
struct DescentGraphs;
// Advances nsteps with the fused step; with `decide`, first chooses pruned or
// full passes for this state (api.cu).  No diagnostics are read back.
int step_advance_decided(dnsbox_ctx *c, void *uh, int nsteps, bool decide);
// N(u) into out on the context's stream, without device selection or host
// synchronisation (api.cu).
int rhs_nonlinear_impl(dnsbox_ctx *ctx, const void *uh, void *out);
// Releases the adjoint descent's captured graphs and stream (adjoint.cu).
void descent_graphs_free(dnsbox_ctx *c);
// Synchronises the context's stream and returns DNSBOX_ERR_TIMEOUT (clearing
// the flag) if a tensor-core pass gave up waiting for its MMAs (api.cu).
int tc_check(dnsbox_ctx *c);
// Applies the schedule cached for the context's device and shape (tune.cu).
void schedule_from_cache(dnsbox_ctx *c);

// ------------------------------------------------------------------ context
struct dnsbox_ctx {
  dnsbox_params p;
  int fp64;                 // 1: complex double, 0: complex float
  size_t cbytes;            // bytes per complex element
  size_t nh, np;            // elements per spectral / physical field
  int nxh;
  cudaStream_t stream = 0;
  char *W1 = nullptr, *W2 = nullptr;     // 6 spectral fields each
  char *ustar = nullptr, *nold = nullptr;
  char *sibuf = nullptr;                 // semi-implicit step: N of the current iterate (3 fields)
  int si_iters = 0;                      // fixed-point iterations of the last semi-implicit step
  int proj_every = 0;                    // project and dealias the state after every step
  char *tw[3] = {nullptr, nullptr, nullptr};
  StepState *st = nullptr;               // device
  double *partials = nullptr;            // device, 2 per finish CTA
  int npartials = 0;
  double *red = nullptr;                 // device scratch for diagnostics
  size_t red_cap = 0;
  int *band = nullptr;                   // band-mode index triples
  int nband = 0;
  dnsbox_diag *ddiag = nullptr;          // device per-step records
  int ddiag_cap = 0;
  double *hstage = nullptr;              // pinned host staging (8 doubles)
  int nspec = 0;
  int ab2_started = 0;
  int cfl_first = 1;                     // reference calls set_time_step before the loop
  int nbatch = 1;                        // boxes of this size advanced together
  size_t fstride = 0;                    // elements between components / work slots (nbatch * nh)
  // The right-hand side keeps its workspace fields (W1, W2) with a padded row
  // pitch: wp complex elements per (z, y) row, a multiple of 128 bytes, so that
  // every row starts on a 128-byte boundary (whole sectors for the strided
  // passes and the x lines, 16-byte aligned tensor-map rows for TMA).
  int wp = 0;
  size_t wstride = 0;                    // elements between workspace slots (nbatch * nz * ny * wp)
  double *d_nu = nullptr;                // per-box viscosity (nbatch > 1) or null
  int ring_cap = 0;                      // device ring of step records: ring_cap steps x nbatch
  long long host_step = 0;               // steps issued so far (ring position)
  const void *force = nullptr;           // fixed spectral forcing (3 fields) or null
  AxisKeep keep[3];                      // pruning rule per axis (x half, y full, z full); a = 0: none
  int prune_ok = 0;                      // the rule prunes something on this grid
  int prune_now = 0;                     // the step in flight uses the pruned passes
  int *cut_flag = nullptr;               // device: the state is nonzero on the cut set
  int tc = 0;                            // DNSBOX_TC_SPLIT: tensor-core strided passes
  void *adft = nullptr;                  // device DFT-64 operands (forward hi, lo, inverse hi, lo)
  int *tc_status = nullptr;              // device flag: an MMA completion wait gave up
  int tc_ctas = 0;                       // persistent grid of the tensor-core passes
  int nsm = 0;                           // streaming multiprocessors of the device
  int tma_on = 0;                        // the right-hand side uses the TMA-staged tensor-core passes
  int tma_box_rows = 32;                 // rows per TMA box of their staged tiles
  int tma_ctas_per_sm = 1;               // resident CTAs per SM of the TMA passes
  // kernel schedule of the right-hand side (chosen by dnsbox_autotune, or the
  // defaults): passes A, B, D 0 = TMA-staged tensor-core kernel, 1 = the
  // cp.async-fed one; pass E1 0 = SIMT, 1 = TMA-staged tensor-core kernel;
  // x pass 0 = default, 1 = block, 2 = warp, 3 = warp with 128 registers
  int sched_tc[4] = {1, 1, 1, 0};         // passes A, B, D: 0 TMA, 1 cp.async, 2 SIMT; E1: 0 SIMT, 1 TMA
  int sched_x = 0;
  char *adj = nullptr;                   // adjoint arena
  size_t adj_bytes = 0;
  char *orbit = nullptr;                 // checkpoints and segment states of the step-transpose chain
  size_t orbit_bytes = 0;
  DescentGraphs *descent = nullptr;      // adjoint descent: captured launch sequences (adjoint.cu)
  // measurement
  int prof_on = 0;
  std::vector<cudaEvent_t> ev_pool;      // pairs
  std::vector<int> ev_kind;
  size_t ev_used = 0;
  int64_t launches[DNSBOX_NPASS] = {0};
  int64_t total_launches = 0;
};

// brackets a launch of pass `kind` with events when profiling is on
struct Prof {
  dnsbox_ctx *c;
  int kind;
  size_t slot;
  int nl;
  Prof(dnsbox_ctx *c_, int k, int nlaunch = 1) : c(c_), kind(k), slot((size_t)-1), nl(nlaunch) {
    c->launches[kind] += nl;
    c->total_launches += nl;
    if (!c->prof_on) return;
    if (2 * (c->ev_used + 1) > c->ev_pool.size()) {
      for (int i = 0; i < 64; ++i) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        c->ev_pool.push_back(e);
      }
      c->ev_kind.resize(c->ev_pool.size() / 2);
    }
    slot = c->ev_used++;
    c->ev_kind[slot] = kind;
    cudaEventRecord(c->ev_pool[2 * slot], c->stream);
  }
  ~Prof() {
    if (slot != (size_t)-1) cudaEventRecord(c->ev_pool[2 * slot + 1], c->stream);
  }
};

// ------------------------------------------------------------ shared kernels
// rhs_Eband (rhs.f90:137-168) over the precomputed band-mode list, stored as
// (offset lo, offset hi, kx) triples; optionally resets the CFL maxima.
// One block per box: u + box * bstride, components fstride apart.
template <typename C>
__global__ void k_eband(const C *u, long long nh, const int *band, int nband, int nx, StepState *st, double s2,
                        int reset_umax, long long bstride = 0) {
  __shared__ double red[32];
  u += (long long)blockIdx.x * bstride;
  st += blockIdx.x;
  double acc = 0.0;
  for (int i = threadIdx.x; i < nband; i += blockDim.x) {
    const long long off = (long long)(unsigned)band[3 * i] | ((long long)band[3 * i + 1] << 32);
    const int kx = band[3 * i + 2];
    const double w = (k_half(kx, nx, 1.0) == 0.0) ? 0.5 : 1.0;   // rhs.f90:151-155
    double e = 0.0;
    for (int c = 0; c < 3; ++c) {
      const C v = u[c * nh + off];
      e += ((double)v.x * v.x + (double)v.y * v.y) * w;
    }
    acc += e;
  }
  double v[1] = {acc};
  block_sum<1>(v, red);
  if (threadIdx.x == 0) {
    st->eband = v[0] * s2;
    if (reset_umax) st->umax[0] = st->umax[1] = st->umax[2] = 0.0;
  }
}

// Sum of n doubles in a fixed order (one block).
template <int NTH>
__global__ void k_sum_scalar(const double *x, int n, double *out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += NTH) acc += x[i];
  double v[1] = {acc};
  block_sum<1>(v, red);
  if (threadIdx.x == 0) *out = v[0];
}

// ------------------------------------------------------------- dispatch
template <typename T> struct Ops {
#define DNSBOX_CASE_STRIDED(NN) \
  case NN: return Launcher<T, NN>::strided(a, inv, ntiles, st);
  static cudaError_t strided(int n, const StridedArgs<T> &a, bool inv, int ntiles, cudaStream_t st) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_STRIDED) }
    return cudaErrorInvalidValue;
  }
#define DNSBOX_CASE_TC(NN) \
  case NN: return Launcher<T, NN>::strided_tc(a, inv, nother, adft, status, nctas, st);
  static cudaError_t strided_tc(int n, const StridedArgs<T> &a, bool inv, int nother, const void *adft,
                                int *status, int nctas, cudaStream_t st) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_TC) }
    return cudaErrorInvalidValue;
  }
#define DNSBOX_CASE_TMA(NN) \
  case NN: return Launcher<T, NN>::strided_tma(a, inv, adft, status, nctas, st);
  static cudaError_t strided_tma(int n, const TmaArgs &a, bool inv, const void *adft, int *status, int nctas,
                                 cudaStream_t st) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_TMA) }
    return cudaErrorInvalidValue;
  }
#define DNSBOX_CASE_HASTMA(NN) \
  case NN: return Launcher<T, NN>::has_tma();
  static bool has_tma(int n) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_HASTMA) }
    return false;
  }
#define DNSBOX_CASE_HASTC(NN) \
  case NN: return Launcher<T, NN>::has_tc();
  static bool has_tc(int n) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_HASTC) }
    return false;
  }
#define DNSBOX_CASE_NL(NN) \
  case NN: return Launcher<T, NN>::xline_nl(a, variant, st);
  static cudaError_t xline_nl(int n, const XlineNLArgs<T> &a, int variant, cudaStream_t st) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_NL) }
    return cudaErrorInvalidValue;
  }
#define DNSBOX_CASE_HASXW(NN) \
  case NN: return Launcher<T, NN>::has_xline_warp();
  static bool has_xline_warp(int n) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_HASXW) }
    return false;
  }
#define DNSBOX_CASE_C2R(NN) \
  case NN: return Launcher<T, NN>::xline_c2r(a, nf, st);
  static cudaError_t xline_c2r(int n, const XlineArgs<T> &a, int nf, cudaStream_t st) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_C2R) }
    return cudaErrorInvalidValue;
  }
#define DNSBOX_CASE_R2C(NN) \
  case NN: return Launcher<T, NN>::xline_r2c(a, nf, st);
  static cudaError_t xline_r2c(int n, const XlineArgs<T> &a, int nf, cudaStream_t st) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_R2C) }
    return cudaErrorInvalidValue;
  }
};

// ---------------------------------------------------------------- helpers
static inline int grid_for(long long n, int threads = 256, int cap = 148 * 16) {
  long long b = (n + threads - 1) / threads;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

static inline char *field(char *base, const dnsbox_ctx *c, int slot) {
  return base + (size_t)slot * c->fstride * c->cbytes;
}
static inline const char *cfield(const char *base, const dnsbox_ctx *c, int slot) {
  return base + (size_t)slot * c->fstride * c->cbytes;
}
// Slot of W1 / W2 in the padded layout of the right-hand side.
static inline char *wfield(char *base, const dnsbox_ctx *c, int slot) {
  return base + (size_t)slot * c->wstride * c->cbytes;
}

// Sets the input (in_ws) and output (out_ws) strides of a strided pass along
// `axis` (2: z, 1: y) to the padded workspace layout; the other side keeps
// the state layout of strided_base.
template <typename T> static void strided_ws(const dnsbox_ctx *c, StridedArgs<T> &a, int axis, bool in_ws,
                                             bool out_ws) {
  const long long wp = c->wp, plane = (long long)c->p.ny * wp, box = plane * c->p.nz;
  const long long rs = axis == 2 ? plane : wp, os = axis == 2 ? wp : plane;
  if (in_ws) {
    a.rowstride = rs;
    a.otherstride = os;
    a.bstride = box;
  }
  if (out_ws) {
    a.rowstride_o = rs;
    a.otherstride_o = os;
    a.bstride_o = box;
  } else if (in_ws) {   // the output keeps the state layout
    a.rowstride_o = axis == 2 ? (long long)c->p.ny * c->nxh : c->nxh;
    a.otherstride_o = axis == 2 ? c->nxh : (long long)c->p.ny * c->nxh;
    a.bstride_o = (long long)c->nh;
  }
}

static inline int ensure_red(dnsbox_ctx *c, size_t ndoubles) {
  if (ndoubles <= c->red_cap) return DNSBOX_OK;
  if (c->red) cudaFree(c->red);
  c->red = nullptr;
  CK(cudaMalloc(&c->red, ndoubles * sizeof(double)));
  c->red_cap = ndoubles;
  return DNSBOX_OK;
}

static inline int ensure_diag(dnsbox_ctx *c, int n) {
  if (n <= c->ddiag_cap) return DNSBOX_OK;
  if (c->ddiag) cudaFree(c->ddiag);
  c->ddiag = nullptr;
  CK(cudaMalloc(&c->ddiag, (size_t)n * sizeof(dnsbox_diag)));
  c->ddiag_cap = n;
  return DNSBOX_OK;
}

template <typename T> static StridedArgs<T> strided_base(const dnsbox_ctx *c, int axis) {
  StridedArgs<T> a;
  memset(&a, 0, sizeof(a));
  a.ncols = c->nxh;
  a.nx = c->p.nx;
  a.alpha_x = c->p.alpha_x;
  a.nbatch = c->nbatch;
  a.bstride = (long long)c->nh;
  if (axis == 2) {  // z: rows kz/z, tiles over y (ky while y is spectral)
    a.tw = reinterpret_cast<const typename CT<T>::type *>(c->tw[2]);
    a.rowstride = (long long)c->p.ny * c->nxh;
    a.otherstride = c->nxh;
    a.alpha_row = c->p.alpha_z;
    a.n_other = c->p.ny;
    a.alpha_other = c->p.alpha_y;
  } else {          // y: rows ky/y, tiles over z
    a.tw = reinterpret_cast<const typename CT<T>::type *>(c->tw[1]);
    a.rowstride = c->nxh;
    a.otherstride = (long long)c->p.ny * c->nxh;
    a.alpha_row = c->p.alpha_y;
  }
  return a;
}

template <typename T>
static void set_job(StridedArgs<T> &a, int j, const void *in1, void *out, double a1 = 1, double b1 = 0,
                    int ks1 = 0, const void *in2 = nullptr, double a2 = 1, double b2 = 0, int ks2 = 0) {
  using C = typename CT<T>::type;
  a.job[j].in1 = reinterpret_cast<const C *>(in1);
  a.job[j].in2 = reinterpret_cast<const C *>(in2);
  a.job[j].out = reinterpret_cast<C *>(out);
  a.job[j].a1 = a1;
  a.job[j].b1 = b1;
  a.job[j].ks1 = ks1;
  a.job[j].a2 = a2;
  a.job[j].b2 = b2;
  a.job[j].ks2 = ks2;
}

// Launches a strided pass.  The column-tile grid follows the kernel's tile
// width: all ceil(nxh / width) tiles, or, when a.kcol prunes, the tiles below
// the cut with the Nyquist column in the first free slot past the cut (or in
// a tile of its own when the cut fills the last low tile); a.koth prunes the
// other axis.
// TMA-staged tensor-core pass (api.cu): `base` is the buffer whose `nslots`
// fields the jobs read (the state for a z pass, W1 for a y pass).
int run_strided_tma(dnsbox_ctx *c, int axis, bool inv, const StridedArgs<float> &a, const void *base, int nslots,
                    int kind);

template <typename T>
static int run_strided(dnsbox_ctx *c, int axis, bool inv, StridedArgs<T> a, int kind = DNSBOX_PASS_OTHER,
                       bool allow_tc = true, const void *tma_base = nullptr, int tma_slots = 0) {
  const int n = axis == 2 ? c->p.nz : c->p.ny;
  const int si = kind == DNSBOX_PASS_Z_INV ? 0 : kind == DNSBOX_PASS_Y_INV ? 1 : kind == DNSBOX_PASS_Y_FWD ? 2
               : kind == DNSBOX_PASS_Z_FWD ? 3 : -1;
  if constexpr (sizeof(T) == 4) {
    // passes A, B, D: TMA unless scheduled on the cp.async or the SIMT kernel;
    // E1: TMA when scheduled
    const bool want = si >= 0 && (si == 3 ? c->sched_tc[3] == 1 : c->sched_tc[si] == 0);
    if (allow_tc && tma_base && c->tc && c->tma_on && Ops<T>::has_tma(n) && want)
      return run_strided_tma(c, axis, inv, a, tma_base, tma_slots, kind);
  }
  const bool simt = si >= 0 && si < 3 && c->sched_tc[si] == 2;
  const bool tc = allow_tc && c->tc && Ops<T>::has_tc(n) && !simt;
  const int width = tc ? 4096 / n : TileCols<T>::v;
  if (a.kcol.a) {
    a.ntx_lo = (a.kcol.a + width - 1) / width;
    const int nt = (c->p.nx / 2) / width;
    // 0: the Nyquist column lies in the low tiles; < 0: it takes the free slot
    // kx = kcol.a of the last low tile; > 0: its own tile follows the low tiles
    a.nyq_tile = nt < a.ntx_lo ? 0 : (a.kcol.a % width ? -1 : nt);
  } else {
    a.ntx_lo = 0;   // full grid
    a.nyq_tile = 0;
  }
  const int nother = a.koth.a ? a.koth.count() : (axis == 2 ? c->p.ny : c->p.nz);
  const int ntiles = strided_ntx(a, width) * nother;
  Prof pr(c, kind);
  if (tc) {
    CK(Ops<T>::strided_tc(n, a, inv, nother, c->adft, c->tc_status, c->tc_ctas, c->stream));
    return DNSBOX_OK;
  }
  CK(Ops<T>::strided(n, a, inv, ntiles, c->stream));
  return DNSBOX_OK;
}

// One output of a batched C2R: sum over terms of in * (a + i b k), with k
// the kx (ks 0), kz (ks 1) or ky (ks 2) wavenumber of the mode, applied in
// the first (z) pass while all three axes are spectral.
struct SpecTerm {
  const void *in;
  double a, b;
  int ks;
};
struct SpecJob {
  SpecTerm t[2];
  int nt;
};

// 3D C2R of nf outputs described by jobs, through W1/W2 in chunks of 6.
// Inputs must not live in W1 or W2 slots [0, 6).
template <typename T>
static int c2r_jobs(dnsbox_ctx *c, int nf, const SpecJob *jobs, void *const *out, double scale) {
  for (int f0 = 0; f0 < nf; f0 += 6) {
    const int m = nf - f0 < 6 ? nf - f0 : 6;
    StridedArgs<T> a = strided_base<T>(c, 2);
    a.njobs = m;
    for (int j = 0; j < m; ++j) {
      const SpecJob &J = jobs[f0 + j];
      set_job<T>(a, j, J.t[0].in, field(c->W1, c, j), J.t[0].a, J.t[0].b, J.t[0].ks,
                 J.nt > 1 ? J.t[1].in : nullptr, J.nt > 1 ? J.t[1].a : 1.0, J.nt > 1 ? J.t[1].b : 0.0,
                 J.nt > 1 ? J.t[1].ks : 0);
    }
    RET(run_strided<T>(c, 2, true, a));
    StridedArgs<T> b = strided_base<T>(c, 1);
    b.njobs = m;
    for (int j = 0; j < m; ++j) set_job<T>(b, j, field(c->W1, c, j), field(c->W2, c, j));
    RET(run_strided<T>(c, 1, true, b));
    XlineArgs<T> x;
    memset(&x, 0, sizeof(x));
    for (int j = 0; j < m; ++j) {
      x.in[j] = field(c->W2, c, j);
      x.out[j] = out[f0 + j];
    }
    x.tw = reinterpret_cast<const typename CT<T>::type *>(c->tw[0]);
    x.nlines = c->p.ny * c->p.nz;
    x.nxh = c->nxh;
    x.scale = scale;
    Prof pr(c, DNSBOX_PASS_OTHER);
    CK(Ops<T>::xline_c2r(c->p.nx, x, m, c->stream));
  }
  return DNSBOX_OK;
}

// 3D C2R of nf spectral fields (in[] -> out[] physical).
template <typename T>
static int c2r_fields(dnsbox_ctx *c, int nf, const void *const *in, void *const *out, double scale) {
  SpecJob jobs[16];
  for (int f = 0; f < nf; ++f) jobs[f] = SpecJob{{{in[f], 1.0, 0.0, 0}, {nullptr, 0, 0, 0}}, 1};
  return c2r_jobs<T>(c, nf, jobs, out, scale);
}

// 3D R2C of nf physical fields, chunks of 6.  Inputs must not live in W1
// slots [0, 6).
template <typename T>
static int r2c_fields(dnsbox_ctx *c, int nf, const void *const *in, void *const *out) {
  for (int f0 = 0; f0 < nf; f0 += 6) {
    const int m = nf - f0 < 6 ? nf - f0 : 6;
    XlineArgs<T> x;
    memset(&x, 0, sizeof(x));
    for (int j = 0; j < m; ++j) {
      x.in[j] = in[f0 + j];
      x.out[j] = field(c->W1, c, j);
    }
    x.tw = reinterpret_cast<const typename CT<T>::type *>(c->tw[0]);
    x.nlines = c->p.ny * c->p.nz;
    x.nxh = c->nxh;
    x.scale = 1.0;
    {
      Prof pr(c, DNSBOX_PASS_OTHER);
      CK(Ops<T>::xline_r2c(c->p.nx, x, m, c->stream));
    }
    StridedArgs<T> b = strided_base<T>(c, 1);
    b.njobs = m;
    for (int j = 0; j < m; ++j) set_job<T>(b, j, field(c->W1, c, j), field(c->W2, c, j));
    RET(run_strided<T>(c, 1, false, b));
    StridedArgs<T> a = strided_base<T>(c, 2);
    a.njobs = m;
    for (int j = 0; j < m; ++j) set_job<T>(a, j, field(c->W2, c, j), out[f0 + j]);
    RET(run_strided<T>(c, 2, false, a));
  }
  return DNSBOX_OK;
}

