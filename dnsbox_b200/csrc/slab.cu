// Slab-decomposed 3D FFT over ranks, one GPU each: dnsbox_slab_*.
//
// The reference distributes every field with p3dfft's one-dimensional
// decomposition (variables.f90:131-157: processor grid 1 x nproc,
// p3dfft_setup, p3dfft_get_dims): in physical space each rank holds a slab of
// nz / P z-planes (x, y whole), in spectral space a slab of ny / P ky rows
// (kz, kx whole); p3dfft_ftran_r2c and p3dfft_btran_c2r (dnsbox.f90:44-46,
// 229-231) transpose between the two with one MPI all-to-all per transform.
//
// Here a rank's transform is two local halves around one all-to-all that the
// caller runs (NCCL over NVLink through torch.distributed, or any collective
// that moves P equal blocks): the library does no communication, so the
// exchange overlaps or batches however the caller's runtime likes, and the
// local halves are the library's own pass kernels.
//
//   forward (z-slab physical -> ky-slab spectral)
//     ftran_local:  x R2C of the nz/P planes, forward y FFT, then the planes'
//                   ky rows are packed by destination rank: block q of `send`
//                   = rows [q ny/P, (q+1) ny/P) of every local plane;
//     (all-to-all: block q of rank r's send -> block r of rank q's recv)
//     ftran_finish: the received blocks, in rank order, are the local ky rows
//                   of all nz planes, i.e. (nz, ny/P, nxh) as they lie; the
//                   forward z FFT writes the spectrum.
//   inverse (ky-slab spectral -> z-slab physical)
//     btran_local:  inverse z FFT into `send`, whose block q is planes
//                   [q nz/P, (q+1) nz/P) of the local ky rows as they lie;
//     (all-to-all)
//     btran_finish: block r of `recv` holds ky rows [r ny/P, ...) of the
//                   local planes; they are unpacked into whole planes, then
//                   inverse y FFT and x C2R.
//
// Layouts (row-major, innermost last; complex elements of the precision):
//   physical slab  (nz/P, ny, nx) real, planes [rank nz/P, (rank+1) nz/P)
//   spectral slab  (nz, ny/P, nx/2+1), ky rows [rank ny/P, (rank+1) ny/P)
//   send / recv    P blocks of nz/P * ny/P * (nx/2+1), block q for rank q
// Transforms are unnormalised, as p3dfft's and dnsbox_r2c / dnsbox_c2r.
//
// rhs_nonlinear over the slabs (rhs.f90:18-135, rhs_Eband :137-168), the
// single-box right-hand side's passes with the exchanges between them:
//   rhs_begin:  band-energy partial of the local ky rows; pass A (inverse z
//               of u, v, w, -dz v, dz u) into five send buffers, whose block
//               q is planes [q nz/P, (q+1) nz/P) as the z FFT writes them;
//   (five all-to-alls; the band energy summed over the ranks)
//   rhs_middle: the received ky rows unpacked into whole planes; pass B
//               (inverse y, the curl assembled by two-term jobs), pass C (the
//               fused x pass: C2R, (omega x u) / N^3, CFL maxima, R2C) and
//               pass D (forward y) on the local planes; N packed by
//               destination into three send buffers;
//   (three all-to-alls; the CFL maxima reduced by max)
//   rhs_finish: pass E1 (forward z) of the received ky-slab and the finish's
//               right-hand-side mode (2/3 mask, projection, band forcing with
//               the global band energy) with the rank's ky offset.
// Unpruned passes throughout.
#include <vector>

#include "internal.cuh"

struct dnsbox_slab {
  int nx, ny, nz, nranks, rank, device, precision;
  int nxh, nzl, nyl;
  size_t blk;        // complex elements of one exchange block
  void *A = nullptr, *B = nullptr;   // scratch, nzl * ny * nxh complex each
  void *tw[3] = {nullptr, nullptr, nullptr};   // exp(-2 pi i j / n), n = nx, ny, nz
  size_t cbytes;
  // right-hand side (dnsbox_slab_rhs_setup)
  bool rhs = false;
  dnsbox_params p;
  void *W = nullptr, *V = nullptr;   // 6 fields of nzl * ny * nxh each
  int *band = nullptr;               // band modes of the local ky rows (offset lo, hi, kx)
  int nband = 0;
  dnsbox::StepState *st = nullptr;   // band energy, CFL maxima, dt of the Heun finishes
  double *rows = nullptr;            // (E, D) sums of the corrector finish's rows, nz * nyl pairs
};

namespace {

int slab_twiddles(dnsbox_slab *s, int axis, int n) {
  std::vector<double> h(2 * (size_t)n);
  for (int j = 0; j < n; ++j) {
    const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)j / (long double)n;
    h[2 * j] = (double)cosl(a);
    h[2 * j + 1] = (double)sinl(a);
  }
  CK(cudaMalloc(&s->tw[axis], (size_t)n * s->cbytes));
  if (s->precision == DNSBOX_FP64) {
    CK(cudaMemcpy(s->tw[axis], h.data(), (size_t)n * 16, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> f(h.size());
    for (size_t i = 0; i < f.size(); ++i) f[i] = (float)h[i];
    CK(cudaMemcpy(s->tw[axis], f.data(), (size_t)n * 8, cudaMemcpyHostToDevice));
  }
  return DNSBOX_OK;
}

void slab_free(dnsbox_slab *s) {
  if (!s) return;
  cudaFree(s->A);
  cudaFree(s->B);
  cudaFree(s->W);
  cudaFree(s->V);
  cudaFree(s->band);
  cudaFree(s->st);
  cudaFree(s->rows);
  for (void *t : s->tw) cudaFree(t);
  delete s;
}

// One plain strided FFT (no multipliers) along an axis of length n with `rows`
// rowstride, `nother` tiles of the other axis otherstride apart.
template <typename T>
int slab_strided(const dnsbox_slab *s, int n, const void *tw, bool inv, const void *in, void *out,
                 long long rowstride, long long otherstride, int nother, cudaStream_t st) {
  using C = typename CT<T>::type;
  StridedArgs<T> a;
  memset(&a, 0, sizeof(a));
  a.njobs = 1;
  a.ncols = s->nxh;
  a.nx = s->nx;
  a.alpha_x = 1.0;
  a.alpha_row = 1.0;
  a.tw = reinterpret_cast<const C *>(tw);
  a.rowstride = rowstride;
  a.otherstride = otherstride;
  a.job[0].in1 = reinterpret_cast<const C *>(in);
  a.job[0].out = reinterpret_cast<C *>(out);
  a.job[0].a1 = 1.0;
  const int ntx = (s->nxh + TileCols<T>::v - 1) / TileCols<T>::v;
  cudaError_t e = Ops<T>::strided(n, a, inv, ntx * nother, st);
  if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "slab %s FFT: %s", inv ? "inverse" : "forward",
                                       cudaGetErrorString(e));
  return DNSBOX_OK;
}

template <typename T>
int slab_xline(const dnsbox_slab *s, bool c2r, const void *in, void *out, cudaStream_t st) {
  using C = typename CT<T>::type;
  XlineArgs<T> x;
  memset(&x, 0, sizeof(x));
  x.in[0] = in;
  x.out[0] = out;
  x.tw = reinterpret_cast<const C *>(s->tw[0]);
  x.nlines = s->nzl * s->ny;
  x.nxh = s->nxh;
  x.scale = 1.0;
  cudaError_t e = c2r ? Ops<T>::xline_c2r(s->nx, x, 1, st) : Ops<T>::xline_r2c(s->nx, x, 1, st);
  if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "slab x-line %s: %s", c2r ? "C2R" : "R2C",
                                       cudaGetErrorString(e));
  return DNSBOX_OK;
}

// Whole planes (nzl, ny, nxh) <-> P blocks (nzl, nyl, nxh): one 2D copy per
// rank, block q holding ky rows [q nyl, (q+1) nyl) of every plane.
int slab_blocks(const dnsbox_slab *s, bool pack, const void *src, void *dst, cudaStream_t st) {
  const size_t row = (size_t)s->nyl * s->nxh * s->cbytes;          // one plane's share of a block
  const size_t plane = (size_t)s->ny * s->nxh * s->cbytes;
  for (int q = 0; q < s->nranks; ++q) {
    const char *from = reinterpret_cast<const char *>(src);
    char *to = reinterpret_cast<char *>(dst);
    cudaError_t e;
    if (pack)
      e = cudaMemcpy2DAsync(to + q * s->blk * s->cbytes, row, from + q * row, plane, row, s->nzl,
                            cudaMemcpyDeviceToDevice, st);
    else
      e = cudaMemcpy2DAsync(to + q * row, plane, from + q * s->blk * s->cbytes, row, row, s->nzl,
                            cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "slab block copy: %s", cudaGetErrorString(e));
  }
  return DNSBOX_OK;
}

template <typename T> int ftran_local(dnsbox_slab *s, const void *phys, void *send, cudaStream_t st) {
  RET(slab_xline<T>(s, false, phys, s->A, st));
  // forward y: rows ky (pitch nxh), one tile row per local plane
  RET(slab_strided<T>(s, s->ny, s->tw[1], false, s->A, s->nranks == 1 ? send : s->B, s->nxh,
                      (long long)s->ny * s->nxh, s->nzl, st));
  if (s->nranks > 1) RET(slab_blocks(s, true, s->B, send, st));
  return DNSBOX_OK;
}

template <typename T> int ftran_finish(dnsbox_slab *s, const void *recv, void *spec, cudaStream_t st) {
  // forward z over the received (nz, nyl, nxh): rows kz, one tile row per local ky
  return slab_strided<T>(s, s->nz, s->tw[2], false, recv, spec, (long long)s->nyl * s->nxh, s->nxh, s->nyl, st);
}

template <typename T> int btran_local(dnsbox_slab *s, const void *spec, void *send, cudaStream_t st) {
  return slab_strided<T>(s, s->nz, s->tw[2], true, spec, send, (long long)s->nyl * s->nxh, s->nxh, s->nyl, st);
}

template <typename T> int btran_finish(dnsbox_slab *s, const void *recv, void *phys, cudaStream_t st) {
  const void *planes = recv;
  if (s->nranks > 1) {
    RET(slab_blocks(s, false, recv, s->A, st));
    planes = s->A;
  }
  RET(slab_strided<T>(s, s->ny, s->tw[1], true, planes, s->B, s->nxh, (long long)s->ny * s->nxh, s->nzl, st));
  return slab_xline<T>(s, true, s->B, phys, st);
}

int slab_begin(const dnsbox_slab *s, const void *a, const void *b) {
  if (!s) return set_err(DNSBOX_ERR_ARG, "null slab");
  if (!a || !b) return set_err(DNSBOX_ERR_ARG, "null pointer");
  CK(cudaSetDevice(s->device));
  return DNSBOX_OK;
}

}  // namespace

extern "C" int dnsbox_slab_create(int nx, int ny, int nz, int nranks, int rank, int precision, int device,
                                  dnsbox_slab **out) {
  if (!out) return set_err(DNSBOX_ERR_ARG, "null argument");
  *out = nullptr;
  if (!dnsbox_supported_size(nx) || !dnsbox_supported_size(ny) || !dnsbox_supported_size(nz))
    return set_err(DNSBOX_ERR_SIZE, "unsupported grid %dx%dx%d", nx, ny, nz);
  if (precision != DNSBOX_FP64 && precision != DNSBOX_FP32)
    return set_err(DNSBOX_ERR_ARG, "precision must be DNSBOX_FP64 or DNSBOX_FP32");
  if (nranks < 1 || rank < 0 || rank >= nranks) return set_err(DNSBOX_ERR_ARG, "rank %d of %d", rank, nranks);
  if (ny % nranks || nz % nranks)
    return set_err(DNSBOX_ERR_ARG, "%d ranks do not divide ny = %d and nz = %d", nranks, ny, nz);
  CK(cudaSetDevice(device));
  dnsbox_slab *s = new dnsbox_slab();
  s->nx = nx;
  s->ny = ny;
  s->nz = nz;
  s->nranks = nranks;
  s->rank = rank;
  s->device = device;
  s->precision = precision;
  s->cbytes = precision == DNSBOX_FP64 ? 16 : 8;
  s->nxh = nx / 2 + 1;
  s->nzl = nz / nranks;
  s->nyl = ny / nranks;
  s->blk = (size_t)s->nzl * s->nyl * s->nxh;
  const size_t bytes = (size_t)s->nzl * ny * s->nxh * s->cbytes;
  int rc = DNSBOX_OK;
  cudaError_t e;
  if ((e = cudaMalloc(&s->A, bytes)) != cudaSuccess || (e = cudaMalloc(&s->B, bytes)) != cudaSuccess) {
    slab_free(s);
    return set_err(DNSBOX_ERR_OOM, "slab scratch (2 x %zu bytes): %s", bytes, cudaGetErrorString(e));
  }
  if ((rc = slab_twiddles(s, 0, nx)) || (rc = slab_twiddles(s, 1, ny)) || (rc = slab_twiddles(s, 2, nz))) {
    slab_free(s);
    return rc;
  }
  *out = s;
  return DNSBOX_OK;
}

extern "C" void dnsbox_slab_destroy(dnsbox_slab *s) {
  if (!s) return;
  cudaSetDevice(s->device);
  slab_free(s);
}

extern "C" int dnsbox_slab_dims(const dnsbox_slab *s, int phys_start[3], int phys_size[3], int spec_start[3],
                                int spec_size[3], size_t *block_elems) {
  if (!s || !phys_start || !phys_size || !spec_start || !spec_size || !block_elems)
    return set_err(DNSBOX_ERR_ARG, "null argument");
  // (z, y, x) order, as the arrays are laid out
  phys_start[0] = s->rank * s->nzl, phys_start[1] = 0, phys_start[2] = 0;
  phys_size[0] = s->nzl, phys_size[1] = s->ny, phys_size[2] = s->nx;
  spec_start[0] = 0, spec_start[1] = s->rank * s->nyl, spec_start[2] = 0;
  spec_size[0] = s->nz, spec_size[1] = s->nyl, spec_size[2] = s->nxh;
  *block_elems = s->blk;
  return DNSBOX_OK;
}

extern "C" int dnsbox_slab_ftran_local(dnsbox_slab *s, const void *phys, void *send, void *stream) {
  RET(slab_begin(s, phys, send));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return s->precision == DNSBOX_FP64 ? ftran_local<double>(s, phys, send, st) : ftran_local<float>(s, phys, send, st);
}

extern "C" int dnsbox_slab_ftran_finish(dnsbox_slab *s, const void *recv, void *spec, void *stream) {
  RET(slab_begin(s, recv, spec));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return s->precision == DNSBOX_FP64 ? ftran_finish<double>(s, recv, spec, st)
                                     : ftran_finish<float>(s, recv, spec, st);
}

extern "C" int dnsbox_slab_btran_local(dnsbox_slab *s, const void *spec, void *send, void *stream) {
  RET(slab_begin(s, spec, send));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return s->precision == DNSBOX_FP64 ? btran_local<double>(s, spec, send, st) : btran_local<float>(s, spec, send, st);
}

extern "C" int dnsbox_slab_btran_finish(dnsbox_slab *s, const void *recv, void *phys, void *stream) {
  RET(slab_begin(s, recv, phys));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return s->precision == DNSBOX_FP64 ? btran_finish<double>(s, recv, phys, st)
                                     : btran_finish<float>(s, recv, phys, st);
}

// ------------------------------------------------------------ right-hand side
namespace {

size_t slab_field(const dnsbox_slab *s) { return (size_t)s->nzl * s->ny * s->nxh; }

template <typename T> const char *fld(const void *base, const dnsbox_slab *s, int f) {
  return reinterpret_cast<const char *>(base) + (size_t)f * slab_field(s) * s->cbytes;
}
template <typename T> char *fld(void *base, const dnsbox_slab *s, int f) {
  return reinterpret_cast<char *>(base) + (size_t)f * slab_field(s) * s->cbytes;
}

// strided arguments of a pass on the ky-slab (z rows) or on the planes (y rows)
template <typename T> StridedArgs<T> slab_pass(const dnsbox_slab *s, bool zslab_rows) {
  StridedArgs<T> a;
  memset(&a, 0, sizeof(a));
  a.ncols = s->nxh;
  a.nx = s->nx;
  a.alpha_x = s->p.alpha_x;
  if (zslab_rows) {   // (nz, nyl, nxh): rows kz, one tile row per local ky
    a.tw = reinterpret_cast<const typename CT<T>::type *>(s->tw[2]);
    a.rowstride = (long long)s->nyl * s->nxh;
    a.otherstride = s->nxh;
    a.alpha_row = s->p.alpha_z;
  } else {            // (nzl, ny, nxh): rows ky, one tile row per local plane
    a.tw = reinterpret_cast<const typename CT<T>::type *>(s->tw[1]);
    a.rowstride = s->nxh;
    a.otherstride = (long long)s->ny * s->nxh;
    a.alpha_row = s->p.alpha_y;
  }
  return a;
}

template <typename T> int slab_run(const dnsbox_slab *s, int n, bool inv, const StridedArgs<T> &a, int nother,
                                   cudaStream_t st) {
  const int ntx = (s->nxh + TileCols<T>::v - 1) / TileCols<T>::v;
  cudaError_t e = Ops<T>::strided(n, a, inv, ntx * nother, st);
  if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "slab right-hand side pass: %s", cudaGetErrorString(e));
  return DNSBOX_OK;
}

template <typename T>
int rhs_begin(dnsbox_slab *s, const void *uh, double *eband, void *send5, cudaStream_t st) {
  using C = typename CT<T>::type;
  const double sc = 1.0 / ((double)s->nx * s->ny * s->nz);
  const size_t F = slab_field(s);   // = nz * nyl * nxh, the ky-slab's field
  k_eband<C><<<1, 256, 0, st>>>(reinterpret_cast<const C *>(uh), (long long)F, s->band, s->nband, s->nx, s->st,
                                sc * sc, 1, 0);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(eband, &s->st->eband, sizeof(double), cudaMemcpyDeviceToDevice, st));
  // pass A: state -> send buffers (rhs.f90:39-65: the spectral curl as multipliers)
  StridedArgs<T> a = slab_pass<T>(s, true);
  a.njobs = 5;
  const char *u = reinterpret_cast<const char *>(uh);
  auto comp = [&](int c) { return u + (size_t)c * F * s->cbytes; };
  set_job<T>(a, 0, comp(0), fld<T>(send5, s, 0));
  set_job<T>(a, 1, comp(1), fld<T>(send5, s, 1));
  set_job<T>(a, 2, comp(2), fld<T>(send5, s, 2));
  set_job<T>(a, 3, comp(1), fld<T>(send5, s, 3), 0.0, -sc, 1);   // -dz v
  set_job<T>(a, 4, comp(0), fld<T>(send5, s, 4), 0.0, sc, 1);    //  dz u
  return slab_run<T>(s, s->nz, true, a, s->nyl, st);
}

template <typename T>
int rhs_middle(dnsbox_slab *s, const void *recv5, double *umax, void *send3, cudaStream_t st) {
  using C = typename CT<T>::type;
  const double sc = 1.0 / ((double)s->nx * s->ny * s->nz);
  // the received ky rows as whole planes (one rank: the buffers are the planes)
  const void *in = recv5;
  if (s->nranks > 1) {
    for (int f = 0; f < 5; ++f) RET(slab_blocks(s, false, fld<T>(recv5, s, f), fld<T>(s->W, s, f), st));
    in = s->W;
  }
  // pass B: inverse y; omega_x = dy w - dz v, omega_y = dz u - dx w, omega_z = dx v - dy u
  StridedArgs<T> b = slab_pass<T>(s, false);
  b.njobs = 6;
  set_job<T>(b, 0, fld<T>(in, s, 0), fld<T>(s->V, s, 0));
  set_job<T>(b, 1, fld<T>(in, s, 1), fld<T>(s->V, s, 1));
  set_job<T>(b, 2, fld<T>(in, s, 2), fld<T>(s->V, s, 2));
  set_job<T>(b, 3, fld<T>(in, s, 2), fld<T>(s->V, s, 3), 0.0, sc, 1, fld<T>(in, s, 3));
  set_job<T>(b, 4, fld<T>(in, s, 4), fld<T>(s->V, s, 4), 1.0, 0.0, 0, fld<T>(in, s, 2), 0.0, -sc, 0);
  set_job<T>(b, 5, fld<T>(in, s, 0), fld<T>(s->V, s, 5), 0.0, -sc, 1, fld<T>(in, s, 1), 0.0, sc, 0);
  RET(slab_run<T>(s, s->ny, true, b, s->nzl, st));
  // pass C: the fused x pass on the local planes
  XlineNLArgs<T> x;
  memset(&x, 0, sizeof(x));
  x.U = reinterpret_cast<const C *>(fld<T>(s->V, s, 0));
  x.V = reinterpret_cast<const C *>(fld<T>(s->V, s, 1));
  x.W = reinterpret_cast<const C *>(fld<T>(s->V, s, 2));
  x.OX = reinterpret_cast<const C *>(fld<T>(s->V, s, 3));
  x.OY = reinterpret_cast<const C *>(fld<T>(s->V, s, 4));
  x.OZ = reinterpret_cast<const C *>(fld<T>(s->V, s, 5));
  x.NX = reinterpret_cast<C *>(fld<T>(s->W, s, 0));
  x.NY = reinterpret_cast<C *>(fld<T>(s->W, s, 1));
  x.NZ = reinterpret_cast<C *>(fld<T>(s->W, s, 2));
  x.tw = reinterpret_cast<const C *>(s->tw[0]);
  x.st = s->st;
  x.lines_per_box = s->ny * s->nzl;
  x.nlines = s->ny * s->nzl;
  x.nxh = s->nxh;
  x.alpha_x = s->p.alpha_x;
  x.s = sc;
  cudaError_t e = Ops<T>::xline_nl(s->nx, x, 0, st);
  if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "slab x pass: %s", cudaGetErrorString(e));
  CK(cudaMemcpyAsync(umax, s->st->umax, 3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
  // pass D: forward y, then N packed by destination rank (one rank: straight
  // into the send buffers)
  void *dout = s->nranks > 1 ? s->V : send3;
  StridedArgs<T> d = slab_pass<T>(s, false);
  d.njobs = 3;
  for (int f = 0; f < 3; ++f) set_job<T>(d, f, fld<T>(s->W, s, f), fld<T>(dout, s, f));
  RET(slab_run<T>(s, s->ny, false, d, s->nzl, st));
  if (s->nranks > 1)
    for (int f = 0; f < 3; ++f) RET(slab_blocks(s, true, fld<T>(s->V, s, f), fld<T>(send3, s, f), st));
  return DNSBOX_OK;
}

template <typename T>
int rhs_finish(dnsbox_slab *s, const void *recv3, const void *uh, const double *eband, void *out, cudaStream_t st,
               int mode = FIN_RHS, void *state = nullptr, double *rows = nullptr) {
  using C = typename CT<T>::type;
  const dnsbox_params &p = s->p;
  // pass E1: forward z of the received ky-slab
  StridedArgs<T> z = slab_pass<T>(s, true);
  z.njobs = 3;
  for (int f = 0; f < 3; ++f) set_job<T>(z, f, fld<T>(recv3, s, f), fld<T>(s->W, s, f));
  RET(slab_run<T>(s, s->nz, false, z, s->nyl, st));
  CK(cudaMemcpyAsync(&s->st->eband, eband, sizeof(double), cudaMemcpyDeviceToDevice, st));
  // pass E2 in right-hand-side mode (rhs.f90:67-133), rows of the rank's ky slab
  FinishArgs<T> f;
  memset(&f, 0, sizeof(f));
  f.n3 = reinterpret_cast<const C *>(s->W);
  f.uin = reinterpret_cast<const C *>(uh);
  f.out = reinterpret_cast<C *>(out);
  f.state = reinterpret_cast<C *>(state);
  f.partials = rows;
  f.st = s->st;
  f.tw = reinterpret_cast<const C *>(s->tw[2]);
  f.nh = (long long)slab_field(s);
  f.nx = s->nx;
  f.ny = s->nyl;
  f.nz = s->nz;
  f.nxh = s->nxh;
  f.ky0 = s->rank * s->nyl;
  f.ny_k = s->ny;
  f.ax = p.alpha_x;
  f.ay = p.alpha_y;
  f.az = p.alpha_z;
  f.nu = p.nu;
  f.Q = p.Q;
  f.Pin = p.Pin;
  f.kcut = p.kCutOff;
  f.cutx = (s->nx / 2.0) * (2.0 * p.alpha_x / 3.0);   // rhs.f90:74-88
  f.cuty = (s->ny / 2.0) * (2.0 * p.alpha_y / 3.0);
  f.cutz = (s->nz / 2.0) * (2.0 * p.alpha_z / 3.0);
  f.sph2 = pow((s->nx / 2.0) * 0.5 * p.alpha_x, 2);
  f.bandlim = p.bandlim;
  f.spherical = p.spherical;
  f.s = 1.0 / ((double)s->nx * s->ny * s->nz);
  f.mode = mode;
  f.kx = AxisKeep{0, s->nx, 0};
  f.ky = AxisKeep{0, s->nyl, 1};
  f.kz = AxisKeep{0, s->nz, 1};
  const int nrows = s->nz * s->nyl;
  const dim3 grid((unsigned)((nrows + 7) / 8), 1);
  switch (mode) {
    case FIN_RHS: k_finish_rows<T, FIN_RHS><<<grid, 256, 0, st>>>(f, nrows); break;
    case FIN_PRED: k_finish_rows<T, FIN_PRED><<<grid, 256, 0, st>>>(f, nrows); break;
    default: k_finish_rows<T, FIN_CORR><<<grid, 256, 0, st>>>(f, nrows); break;
  }
  CK(cudaGetLastError());
  return DNSBOX_OK;
}

int rhs_begin_check(const dnsbox_slab *s, const void *a, const void *b, const void *c) {
  if (!s) return set_err(DNSBOX_ERR_ARG, "null slab");
  if (!s->rhs) return set_err(DNSBOX_ERR_STATE, "dnsbox_slab_rhs_setup has not been called");
  if (!a || !b || !c) return set_err(DNSBOX_ERR_ARG, "null pointer");
  CK(cudaSetDevice(s->device));
  return DNSBOX_OK;
}

}  // namespace

extern "C" int dnsbox_slab_rhs_setup(dnsbox_slab *s, const dnsbox_params *p) {
  if (!s || !p) return set_err(DNSBOX_ERR_ARG, "null argument");
  if (p->nx != s->nx || p->ny != s->ny || p->nz != s->nz)
    return set_err(DNSBOX_ERR_ARG, "grid %dx%dx%d is not the slab's %dx%dx%d", p->nx, p->ny, p->nz, s->nx, s->ny,
                   s->nz);
  if (!(p->nu >= 0.0) || !(p->alpha_x > 0) || !(p->alpha_y > 0) || !(p->alpha_z > 0))
    return set_err(DNSBOX_ERR_ARG, "invalid physical parameter");
  CK(cudaSetDevice(s->device));
  s->p = *p;
  // buffers once (a repeated set-up, or one after a failed allocation, keeps
  // what is there and allocates the rest)
  const size_t bytes = 6 * slab_field(s) * s->cbytes;
  if (!s->W) CK(cudaMalloc(&s->W, bytes));
  if (!s->V) CK(cudaMalloc(&s->V, bytes));
  if (!s->st) {
    CK(cudaMalloc(&s->st, sizeof(dnsbox::StepState)));
    CK(cudaMemset(s->st, 0, sizeof(dnsbox::StepState)));
  }
  if (!s->rows) CK(cudaMalloc(&s->rows, 2 * (size_t)s->nz * s->nyl * sizeof(double)));
  // band modes |k| <= kCutOff among the local ky rows (as dnsbox_create builds them)
  cudaFree(s->band);
  s->band = nullptr;
  s->nband = 0;
  std::vector<int> band;
  if (p->bandlim) {
    const int ky0 = s->rank * s->nyl;
    for (int kz = 0; kz < s->nz; ++kz)
      for (int yl = 0; yl < s->nyl; ++yl)
        for (int kx = 0; kx < s->nxh; ++kx) {
          const double a = k_half(kx, s->nx, p->alpha_x), b = k_full(ky0 + yl, s->ny, p->alpha_y),
                       c = k_full(kz, s->nz, p->alpha_z);
          if (sqrt(a * a + b * b + c * c) > p->kCutOff) continue;
          const long long off = ((long long)kz * s->nyl + yl) * s->nxh + kx;
          band.push_back((int)(off & 0xffffffffLL));
          band.push_back((int)(off >> 32));
          band.push_back(kx);
        }
  }
  s->nband = (int)band.size() / 3;
  if (s->nband) {
    CK(cudaMalloc(&s->band, band.size() * sizeof(int)));
    CK(cudaMemcpy(s->band, band.data(), band.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  s->rhs = true;
  return DNSBOX_OK;
}

extern "C" int dnsbox_slab_rhs_begin(dnsbox_slab *s, const void *uh, double *eband_dev, void *send5, void *stream) {
  RET(rhs_begin_check(s, uh, eband_dev, send5));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return s->precision == DNSBOX_FP64 ? rhs_begin<double>(s, uh, eband_dev, send5, st)
                                     : rhs_begin<float>(s, uh, eband_dev, send5, st);
}

extern "C" int dnsbox_slab_rhs_middle(dnsbox_slab *s, const void *recv5, double *umax_dev, void *send3,
                                      void *stream) {
  RET(rhs_begin_check(s, recv5, umax_dev, send3));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return s->precision == DNSBOX_FP64 ? rhs_middle<double>(s, recv5, umax_dev, send3, st)
                                     : rhs_middle<float>(s, recv5, umax_dev, send3, st);
}

extern "C" int dnsbox_slab_rhs_finish(dnsbox_slab *s, const void *recv3, const void *uh, const double *eband_dev,
                                      void *out, void *stream) {
  RET(rhs_begin_check(s, recv3, eband_dev, out));
  if (!uh) return set_err(DNSBOX_ERR_ARG, "null pointer");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return s->precision == DNSBOX_FP64 ? rhs_finish<double>(s, recv3, uh, eband_dev, out, st)
                                     : rhs_finish<float>(s, recv3, uh, eband_dev, out, st);
}

// dt of the finishes that follow on the stream (a kernel argument: no host
// staging to keep alive)
__global__ void k_slab_set_dt(dnsbox::StepState *st, double dt) { st->dt = dt; }

// The rank's (E, D) sums: the corrector finish's row pairs added in a fixed
// order (one block), unscaled, for the caller's sum over the ranks.
__global__ void k_slab_row_sums(const double *rows, int n, double *ed) {
  __shared__ double red[2 * 32];
  double e = 0.0, d = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    e += rows[2 * i];
    d += rows[2 * i + 1];
  }
  double v[2] = {e, d};
  dnsbox::block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    ed[0] = v[0];
    ed[1] = v[1];
  }
}

// IF-Heun over the slabs (dnsboxheun.f90:88-126): the predictor's finish
// u* = IF (u + dt N(u)) into `out`, the corrector's u <- (IF u + u*) / 2 +
// dt/2 N(u*) in place in `state` (uin = u*), with the rank's unscaled (E, D)
// sums of the new state into ed_dev (state_kinetic / state_dissipation in
// Parseval form: E = s^2 sum, D = nu s^2 sum after the sum over the ranks).
extern "C" int dnsbox_slab_heun_finish(dnsbox_slab *s, const void *recv3, const void *uin_dev,
                                       const double *eband_dev, int corrector, double dt, void *out_dev,
                                       double *ed_dev, void *cuda_stream) {
  RET(rhs_begin_check(s, recv3, eband_dev, out_dev));
  if (!uin_dev) return set_err(DNSBOX_ERR_ARG, "null pointer");
  if (!(dt > 0.0) || !isfinite(dt)) return set_err(DNSBOX_ERR_ARG, "dt must be positive and finite");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(cuda_stream);
  k_slab_set_dt<<<1, 1, 0, st>>>(s->st, dt);
  CK(cudaGetLastError());
  const int mode = corrector ? FIN_CORR : FIN_PRED;
  void *out = corrector ? nullptr : out_dev, *state = corrector ? out_dev : nullptr;
  double *rows = corrector && ed_dev ? s->rows : nullptr;
  RET(s->precision == DNSBOX_FP64 ? rhs_finish<double>(s, recv3, uin_dev, eband_dev, out, st, mode, state, rows)
                                  : rhs_finish<float>(s, recv3, uin_dev, eband_dev, out, st, mode, state, rows));
  if (rows) {
    k_slab_row_sums<<<1, 256, 0, st>>>(rows, s->nz * s->nyl, ed_dev);
    CK(cudaGetLastError());
  }
  return DNSBOX_OK;
}
