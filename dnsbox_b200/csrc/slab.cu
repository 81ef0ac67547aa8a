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
#include <vector>

#include "internal.cuh"

struct dnsbox_slab {
  int nx, ny, nz, nranks, rank, device, precision;
  int nxh, nzl, nyl;
  size_t blk;        // complex elements of one exchange block
  void *A = nullptr, *B = nullptr;   // scratch, nzl * ny * nxh complex each
  void *tw[3] = {nullptr, nullptr, nullptr};   // exp(-2 pi i j / n), n = nx, ny, nz
  size_t cbytes;
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
