// Allocation-free 3D C2R: dnsbox_c2r_noalloc.
//
// Some callers cannot call cudaMalloc: a host program whose device memory is
// handed to its own pool or arena at start-up (and must not be bypassed), or a
// time-critical loop in which allocating is not allowed.  They cannot create a
// dnsbox_ctx either, because dnsbox_create allocates the context's workspace.
// This entry point runs the same three passes as dnsbox_c2r (inverse z and y
// FFTs, then the x-line C2R) without a context: the two intermediate spectral
// fields live in a file-scope static __device__ array of kScratchBytes, and the
// twiddle tables in a second static __device__ array.  Every GPU that loads the
// library holds both arrays until the process exits.
//
// Set-up: the first call on a device (with that device current) resolves the
// arrays' device addresses with cudaGetSymbolAddress and fills the twiddle
// tables; later calls on that device reuse them.  Make that first call before
// any stream capture.  Every call resolves the scratch address again (a host
// lookup, no allocation); when it differs from the one set up -- the module was
// reloaded after cudaDeviceReset or a primary-context teardown -- the set-up
// runs again, so the first call after such a reset must also come before any
// stream capture.  Host code never hands the arrays' names to a kernel: in host
// code they are stand-ins, not device addresses.
//
// Every call shares the scratch array and leaves its contents behind.  Nothing
// in it has to start at zero: each pass writes every element the next pass
// reads.  Calls that overlap on the GPU (other streams, other host threads)
// race on the array; serialise them.
#include <mutex>

#include "internal.cuh"

namespace {

constexpr size_t kScratchBytes = size_t(8) << 20;   // two spectral fields at most
constexpr int kTwLens[] = {8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 512, 1024};
constexpr int kTwTotal = 8 + 12 + 16 + 24 + 32 + 48 + 64 + 96 + 128 + 192 + 256 + 512 + 1024;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];
static __device__ __align__(256) double2 g_tw64[kTwTotal];
static __device__ __align__(256) float2 g_tw32[kTwTotal];

struct DeviceSetup {
  bool done = false;
  unsigned char *scratch = nullptr;   // device address of g_scratch
  double2 *tw64 = nullptr;
  float2 *tw32 = nullptr;
};
DeviceSetup g_dev[kMaxDevices];
std::mutex g_mu;

int tw_offset(int n) {
  int off = 0;
  for (int len : kTwLens) {
    if (len == n) return off;
    off += len;
  }
  return -1;
}

// Once per device (and again after the module was reloaded), with the device
// current: resolve the symbols and fill the twiddle tables exp(-2 pi i j / n).
int setup_device(int dev, DeviceSetup **out) {
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceSetup &d = g_dev[dev];
  if (d.done) {
    unsigned char *now = nullptr;
    cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&now), g_scratch);
    if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    if (now != d.scratch) d.done = false;   // a new module instance: its twiddle tables are unfilled
  }
  if (!d.done) {
    cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&d.scratch), g_scratch);
    if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    e = cudaGetSymbolAddress(reinterpret_cast<void **>(&d.tw64), g_tw64);
    if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "cudaGetSymbolAddress(tw64): %s", cudaGetErrorString(e));
    e = cudaGetSymbolAddress(reinterpret_cast<void **>(&d.tw32), g_tw32);
    if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "cudaGetSymbolAddress(tw32): %s", cudaGetErrorString(e));
    static double2 h64[kTwTotal];   // host staging, static: the set-up allocates nothing
    static float2 h32[kTwTotal];
    int off = 0;
    for (int n : kTwLens) {
      for (int j = 0; j < n; ++j) {
        const long double a = -2.0L * 3.141592653589793238462643383279502884L * j / (long double)n;
        h64[off + j] = make_double2((double)cosl(a), (double)sinl(a));
        h32[off + j] = make_float2((float)cosl(a), (float)sinl(a));
      }
      off += n;
    }
    e = cudaMemcpy(d.tw64, h64, sizeof(double2) * kTwTotal, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "twiddle upload: %s", cudaGetErrorString(e));
    e = cudaMemcpy(d.tw32, h32, sizeof(float2) * kTwTotal, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "twiddle upload: %s", cudaGetErrorString(e));
    d.done = true;
  }
  *out = &d;
  return DNSBOX_OK;
}

template <typename T>
int c2r_noalloc(int nx, int ny, int nz, const void *spec, void *phys, cudaStream_t st, const DeviceSetup &d) {
  using C = typename CT<T>::type;
  const C *tw = reinterpret_cast<const C *>(sizeof(T) == 8 ? (const void *)d.tw64 : (const void *)d.tw32);
  const int nxh = nx / 2 + 1;
  const size_t nh = (size_t)nz * ny * nxh;
  C *bufA = reinterpret_cast<C *>(d.scratch);
  C *bufB = bufA + nh;
  const int ntx = (nxh + TileCols<T>::v - 1) / TileCols<T>::v;
  // inverse z: spec -> A
  StridedArgs<T> a;
  memset(&a, 0, sizeof(a));
  a.njobs = 1;
  a.ncols = nxh;
  a.nx = nx;
  a.alpha_x = 1.0;
  a.alpha_row = 1.0;
  a.tw = tw + tw_offset(nz);
  a.rowstride = (long long)ny * nxh;
  a.otherstride = nxh;
  a.job[0].in1 = reinterpret_cast<const C *>(spec);
  a.job[0].out = bufA;
  a.job[0].a1 = 1.0;
  cudaError_t e = Ops<T>::strided(nz, a, true, ntx * ny, st);
  if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "inverse z pass: %s", cudaGetErrorString(e));
  // inverse y: A -> B
  StridedArgs<T> b = a;
  b.tw = tw + tw_offset(ny);
  b.rowstride = nxh;
  b.otherstride = (long long)ny * nxh;
  b.job[0].in1 = bufA;
  b.job[0].out = bufB;
  e = Ops<T>::strided(ny, b, true, ntx * nz, st);
  if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "inverse y pass: %s", cudaGetErrorString(e));
  // x-line C2R: B -> phys
  XlineArgs<T> x;
  memset(&x, 0, sizeof(x));
  x.in[0] = bufB;
  x.out[0] = phys;
  x.tw = tw + tw_offset(nx);
  x.nlines = ny * nz;
  x.nxh = nxh;
  x.scale = 1.0;
  e = Ops<T>::xline_c2r(nx, x, 1, st);
  if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "x-line C2R pass: %s", cudaGetErrorString(e));
  return DNSBOX_OK;
}

}  // namespace

extern "C" int dnsbox_c2r_noalloc(int nx, int ny, int nz, int precision, const void *spec_dev, void *phys_dev,
                                  void *cuda_stream) {
  if (!spec_dev || !phys_dev) return set_err(DNSBOX_ERR_ARG, "null pointer");
  if (precision != DNSBOX_FP64 && precision != DNSBOX_FP32)
    return set_err(DNSBOX_ERR_ARG, "precision must be DNSBOX_FP64 or DNSBOX_FP32");
  if (!dnsbox_supported_size(nx) || !dnsbox_supported_size(ny) || !dnsbox_supported_size(nz))
    return set_err(DNSBOX_ERR_SIZE, "unsupported grid %dx%dx%d", nx, ny, nz);
  const size_t need = 2 * (size_t)nz * ny * (nx / 2 + 1) * (precision == DNSBOX_FP64 ? 16 : 8);
  if (need > kScratchBytes)
    return set_err(DNSBOX_ERR_SIZE,
                   "grid %dx%dx%d needs %zu bytes of scratch; dnsbox_c2r_noalloc holds %zu (use dnsbox_c2r)", nx, ny,
                   nz, need, kScratchBytes);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_err(DNSBOX_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return set_err(DNSBOX_ERR_ARG, "device ordinal %d out of range", dev);
  DeviceSetup *d = nullptr;
  int rc = setup_device(dev, &d);
  if (rc != DNSBOX_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(cuda_stream);
  return precision == DNSBOX_FP64 ? c2r_noalloc<double>(nx, ny, nz, spec_dev, phys_dev, st, *d)
                                  : c2r_noalloc<float>(nx, ny, nz, spec_dev, phys_dev, st, *d);
}
