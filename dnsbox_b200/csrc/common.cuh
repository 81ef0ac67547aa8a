// Common device types and helpers for the dnsbox B200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dnsbox {

template <typename T> struct CT;
template <> struct CT<double> { using type = double2; };
template <> struct CT<float> { using type = float2; };

template <typename C> __host__ __device__ __forceinline__ C mkc(decltype(C{}.x) re, decltype(C{}.x) im) {
  C c;
  c.x = re;
  c.y = im;
  return c;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mkc<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mkc<C>(a.x - b.x, a.y - b.y); }
// Single precision: one paired FP32 instruction (add/sub .f32x2, sm_100) for
// both parts, each rounded to nearest as a scalar add would be.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "add.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mkc<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  return mkc<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) { return mkc<C>(a.x * s, a.y * s); }
// forward transform uses -i, inverse +i
template <bool INV, typename C> __device__ __forceinline__ C mul_i(C a) {
  return INV ? mkc<C>(-a.y, a.x) : mkc<C>(a.y, -a.x);
}

// Integrating factor exp(x), evaluated in FP64 and rounded once to the
// state's precision: it multiplies the whole state every step, so its error
// goes straight into the velocity (single-precision expf, up to 2 ulp, moved
// the 512^3 FP32 run's velocity error against FP64 from 0.7e-6 to 1.6e-6).
template <typename T> __device__ __forceinline__ T if_exp(double x) { return T(exp(x)); }

// Wavenumber of an index along a full axis of length n (variables.f90:242-262):
// 0..n/2-1 -> itself, n/2 (Nyquist) -> 0, n/2+1..n-1 -> index - n.
__host__ __device__ __forceinline__ double k_full(int idx, int n, double alpha) {
  int h = n >> 1;
  return (idx < h ? idx : (idx == h ? 0 : idx - n)) * alpha;
}
// Half axis 0..n/2 (variables.f90:226-229): index n/2 -> 0.
__host__ __device__ __forceinline__ double k_half(int idx, int n, double alpha) {
  return (idx == (n >> 1) ? 0 : idx) * alpha;
}

// Non-negative double max through the integer ordering of IEEE-754 bits.
__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

template <typename T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <typename T> __device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum of NV doubles into out[0..NV) (valid in thread 0).  scratch
// must hold 32*NV doubles.  All threads must call it.
template <int NV> __device__ __forceinline__ void block_sum(double (&v)[NV], double *scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = warp_sum(v[i]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < NV; ++i) scratch[i * 32 + wid] = v[i];
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double x = lane < nw ? scratch[i * 32 + lane] : 0.0;
      v[i] = warp_sum(x);
    }
  }
  __syncthreads();
}

}  // namespace dnsbox
