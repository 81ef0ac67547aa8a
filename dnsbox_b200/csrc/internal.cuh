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

// ------------------------------------------------------------- dispatch
template <typename T> struct Ops {
#define DNSBOX_CASE_STRIDED(NN) \
  case NN: return Launcher<T, NN>::strided(a, inv, ntiles, st);
  static cudaError_t strided(int n, const StridedArgs<T> &a, bool inv, int ntiles, cudaStream_t st) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_STRIDED) }
    return cudaErrorInvalidValue;
  }
#define DNSBOX_CASE_NL(NN) \
  case NN: return Launcher<T, NN>::xline_nl(a, st);
  static cudaError_t xline_nl(int n, const XlineNLArgs<T> &a, cudaStream_t st) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_NL) }
    return cudaErrorInvalidValue;
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
#define DNSBOX_CASE_FINC(NN) \
  case NN: return Launcher<T, NN>::zfinish_cols();
  static int zfinish_cols(int n) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_FINC) }
    return 1;
  }
#define DNSBOX_CASE_FIN(NN) \
  case NN: return Launcher<T, NN>::zfinish(a, nb, st);
  static cudaError_t zfinish(int n, const FinishArgs<T> &a, int nb, cudaStream_t st) {
    switch (n) { DNSBOX_SIZES(DNSBOX_CASE_FIN) }
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

static inline char *field(char *base, const dnsbox_ctx *c, int slot) { return base + (size_t)slot * c->nh * c->cbytes; }
static inline const char *cfield(const char *base, const dnsbox_ctx *c, int slot) {
  return base + (size_t)slot * c->nh * c->cbytes;
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
  if (axis == 2) {  // z: rows kz/z, tiles over y
    a.tw = reinterpret_cast<const typename CT<T>::type *>(c->tw[2]);
    a.rowstride = (long long)c->p.ny * c->nxh;
    a.otherstride = c->nxh;
    a.alpha_row = c->p.alpha_z;
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

template <typename T>
static int run_strided(dnsbox_ctx *c, int axis, bool inv, const StridedArgs<T> &a,
                       int kind = DNSBOX_PASS_OTHER) {
  const int ntx = (c->nxh + TileCols<T>::v - 1) / TileCols<T>::v;
  const int nother = axis == 2 ? c->p.ny : c->p.nz;
  const int n = axis == 2 ? c->p.nz : c->p.ny;
  Prof pr(c, kind);
  CK(Ops<T>::strided(n, a, inv, ntx * nother, c->stream));
  return DNSBOX_OK;
}

// 3D C2R of nf spectral fields (in[] -> out[] physical), through W1/W2.
// Inputs must not live in W1 slots [0, nf) or W2 slots [0, nf).
template <typename T>
static int c2r_fields(dnsbox_ctx *c, int nf, const void *const *in, void *const *out, double scale) {
  StridedArgs<T> a = strided_base<T>(c, 2);
  a.njobs = nf;
  for (int f = 0; f < nf; ++f) set_job<T>(a, f, in[f], field(c->W1, c, f));
  RET(run_strided<T>(c, 2, true, a));
  StridedArgs<T> b = strided_base<T>(c, 1);
  b.njobs = nf;
  for (int f = 0; f < nf; ++f) set_job<T>(b, f, field(c->W1, c, f), field(c->W2, c, f));
  RET(run_strided<T>(c, 1, true, b));
  XlineArgs<T> x;
  memset(&x, 0, sizeof(x));
  for (int f = 0; f < nf; ++f) {
    x.in[f] = field(c->W2, c, f);
    x.out[f] = out[f];
  }
  x.tw = reinterpret_cast<const typename CT<T>::type *>(c->tw[0]);
  x.nlines = c->p.ny * c->p.nz;
  x.nxh = c->nxh;
  x.scale = scale;
  Prof pr(c, DNSBOX_PASS_OTHER);
  CK(Ops<T>::xline_c2r(c->p.nx, x, nf, c->stream));
  return DNSBOX_OK;
}

// 3D R2C of nf physical fields.  Inputs must not live in W1 slots [0, nf).
template <typename T>
static int r2c_fields(dnsbox_ctx *c, int nf, const void *const *in, void *const *out) {
  XlineArgs<T> x;
  memset(&x, 0, sizeof(x));
  for (int f = 0; f < nf; ++f) {
    x.in[f] = in[f];
    x.out[f] = field(c->W1, c, f);
  }
  x.tw = reinterpret_cast<const typename CT<T>::type *>(c->tw[0]);
  x.nlines = c->p.ny * c->p.nz;
  x.nxh = c->nxh;
  x.scale = 1.0;
  {
    Prof pr(c, DNSBOX_PASS_OTHER);
    CK(Ops<T>::xline_r2c(c->p.nx, x, nf, c->stream));
  }
  StridedArgs<T> b = strided_base<T>(c, 1);
  b.njobs = nf;
  for (int f = 0; f < nf; ++f) set_job<T>(b, f, field(c->W1, c, f), field(c->W2, c, f));
  RET(run_strided<T>(c, 1, false, b));
  StridedArgs<T> a = strided_base<T>(c, 2);
  a.njobs = nf;
  for (int f = 0; f < nf; ++f) set_job<T>(a, f, field(c->W2, c, f), out[f]);
  RET(run_strided<T>(c, 2, false, a));
  return DNSBOX_OK;
}

