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

// Separately rounded products and sums (never contracted into an FMA), for
// the expressions whose last bit decides an integer on the reference's
// separate-operation arithmetic: the spectral integrals behind the cut-off
// index, the stress sums of the LFACTOR iteration, the drag law of u*.
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
// Quotients a / b for one divisor b, each rounded as the IEEE division
// rounds it, without a division per quotient.  In single precision the
// quotient is the float rounding of a times the double reciprocal of b.  That
// product is within 2^-52 (relative) of a/b, while a/b lies more than 2^-49
// (relative) from every midpoint between two floats: a midpoint m has an odd
// 25-bit significand, so a - m*b is a nonzero multiple of 2^-25 ulp(a).  Both
// therefore round to the same float.  Branch-free, unlike the division's
// special-operand paths.  In double precision it is the division itself.
template <typename R> struct RecipDiv;
template <> struct RecipDiv<float> {
  double y;
  __device__ explicit RecipDiv(float b) : y(1.0 / (double)b) {}
  __device__ float operator()(float a) const { return __double2float_rn(__dmul_rn((double)a, y)); }
};
template <> struct RecipDiv<double> {
  double b;
  __device__ explicit RecipDiv(double b_) : b(b_) {}
  __device__ double operator()(double a) const { return a / b; }
};
// Correctly rounded single-precision transcendentals (evaluated in double,
// rounded once) for the same per-point values: the cut-off index's LOG10 /
// LOG, the LFACTOR exponentials and wind-direction cosines, and WAVNU2's
// dispersion relation.  The CPU oracle evaluates them the same way, so equal
// inputs give equal integer decisions.  In double precision they are the
// functions themselves.
__device__ __forceinline__ float crlog10(float x) { return (float)log10((double)x); }
__device__ __forceinline__ double crlog10(double x) { return log10(x); }
__device__ __forceinline__ float crlog(float x) { return (float)log((double)x); }
__device__ __forceinline__ double crlog(double x) { return log(x); }
__device__ __forceinline__ float crexp(float x) { return (float)exp((double)x); }
__device__ __forceinline__ double crexp(double x) { return exp(x); }
__device__ __forceinline__ float crcos(float x) { return (float)cos((double)x); }
__device__ __forceinline__ double crcos(double x) { return cos(x); }
__device__ __forceinline__ float crsin(float x) { return (float)sin((double)x); }
__device__ __forceinline__ double crsin(double x) { return sin(x); }
__device__ __forceinline__ float crtanh(float x) { return (float)tanh((double)x); }
__device__ __forceinline__ double crtanh(double x) { return tanh(x); }
__device__ __forceinline__ float crcosh(float x) { return (float)cosh((double)x); }
__device__ __forceinline__ double crcosh(double x) { return cosh(x); }
__device__ __forceinline__ float crsinh(float x) { return (float)sinh((double)x); }
__device__ __forceinline__ double crsinh(double x) { return sinh(x); }

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
