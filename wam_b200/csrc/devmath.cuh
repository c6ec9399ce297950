// Precision-generic device math and warp reductions (float -> CUDA single
// precision library functions, double -> double precision ones).
#pragma once
#include <cuda_runtime.h>
#include <limits>

namespace wamgpu {

__device__ __forceinline__ float dsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double dsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float dexp(float x) { return expf(x); }
__device__ __forceinline__ double dexp(double x) { return exp(x); }
__device__ __forceinline__ float dlog(float x) { return logf(x); }
__device__ __forceinline__ double dlog(double x) { return log(x); }
__device__ __forceinline__ float dlog10(float x) { return log10f(x); }
__device__ __forceinline__ double dlog10(double x) { return log10(x); }
__device__ __forceinline__ float dpow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double dpow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float dsin(float x) { return sinf(x); }
__device__ __forceinline__ double dsin(double x) { return sin(x); }
__device__ __forceinline__ float dcos(float x) { return cosf(x); }
__device__ __forceinline__ double dcos(double x) { return cos(x); }
__device__ __forceinline__ float dtanh(float x) { return tanhf(x); }
__device__ __forceinline__ double dtanh(double x) { return tanh(x); }
__device__ __forceinline__ float dsinh(float x) { return sinhf(x); }
__device__ __forceinline__ double dsinh(double x) { return sinh(x); }
__device__ __forceinline__ float dcosh(float x) { return coshf(x); }
__device__ __forceinline__ double dcosh(double x) { return cosh(x); }
__device__ __forceinline__ float datan2(float y, float x) { return atan2f(y, x); }
__device__ __forceinline__ double datan2(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ float dabs(float x) { return fabsf(x); }
__device__ __forceinline__ double dabs(double x) { return fabs(x); }
// Fortran MAX/MIN semantics for ordered operands
// a / b through the hardware reciprocal path for FP32 (at most 2 ulp,
// |b| in [2^-126, 2^126]); the precise division for FP64.  Used where the
// divisor is bounded, as max(1, ...) is.
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }

template <typename R> __device__ __forceinline__ R dmax(R a, R b) { return a < b ? b : a; }
template <typename R> __device__ __forceinline__ R dmin(R a, R b) { return b < a ? b : a; }

template <typename R> __device__ __forceinline__ R warp_sum(R v) {
  for (int o = 16; o > 0; o >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Four consecutive reals from a 16-byte aligned address.
template <typename R> struct Quad { R a, b, c, d; };
__device__ __forceinline__ Quad<float> ld4(const float* p) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ Quad<double> ld4(const double* p) {
  const double2 u = *reinterpret_cast<const double2*>(p), v = *reinterpret_cast<const double2*>(p + 2);
  return {u.x, u.y, v.x, v.y};
}
template <typename R> __device__ __forceinline__ R warp_max(R v) {
  for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace wamgpu
