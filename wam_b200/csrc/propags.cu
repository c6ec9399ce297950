// PROPAGS stencil and CHECK_CFL coefficient extrema (compiled with
// -fmad=false so the coefficient arithmetic rounds like the reference).
#include "propags.cuh"
#include "kernels.hpp"

namespace wamgpu {

template <typename R>
__global__ void __launch_bounds__(128) propags_kernel(const PropArgs<R> A, const R* __restrict__ f1, int ld1,
                                                      R* __restrict__ f3, int ld3) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = blockIdx.y;
  if (i >= A.nsea) return;
  const PropCore<R> P(A);
  const int KL = A.KL, ML = A.ML;
  const bool cur = A.variant == V_CART_DEEP_CUR || A.variant == V_CART_SHALLOW_CUR || A.variant == V_SPHER_DEEP_CURR ||
                   A.variant == V_SPHER_SHALLOW_CURR;
  const size_t plane = (size_t)ld1 * KL;
  auto F = [&](int p1, int k, int mm) -> R { return p1 == 0 ? R(0) : __ldg(&f1[(p1 - 1) + (size_t)ld1 * k + plane * mm]); };
  const int s0 = P.klat(i, 0, 0), n0 = P.klat(i, 1, 0), w0 = P.klon(i, 0), e0 = P.klon(i, 1);
  const int s1 = A.reduced ? P.klat(i, 0, 1) : 0, n1 = A.reduced ? P.klat(i, 1, 1) : 0;
  const bool theta = A.refr_d || A.spherical;
  const int mm = (m == 0) ? 0 : m - 1, mp = (m == ML - 1) ? ML - 1 : m + 1;
  R fkm = F(i + 1, KL - 1, m), fk = F(i + 1, 0, m);
  for (int k = 0; k < KL; ++k) {
    const int kp = (k + 1 == KL) ? 0 : k + 1;
    R fkp = F(i + 1, kp, m);
    const Coefs<R> c = P.coef(i, k, m);
    R v;
    if (!cur) {
      const R sn = __ldg(&A.SINTH[k]), cs = __ldg(&A.COSTH[k]);
      const int lat = (cs >= R(0.)) ? s0 : n0, lon = (sn >= R(0.)) ? w0 : e0;
      v = c.sum * fk + c.lat11 * F(lat, k, m) + c.lon1 * F(lon, k, m);
      if (theta) v = v + c.th1 * fkp + c.th2 * fkm;
      if (A.reduced) v = v + c.lat12 * F((cs >= R(0.)) ? s1 : n1, k, m);
    } else {
      v = c.sum * fk + c.lat21 * F(n0, k, m) + c.lat11 * F(s0, k, m) + c.lon2 * F(e0, k, m) + c.lon1 * F(w0, k, m) +
          c.th1 * fkp + c.th2 * fkm + c.sg1 * F(i + 1, k, mp) + c.sg2 * F(i + 1, k, mm);
      if (A.reduced) v = v + c.lat22 * F(n1, k, m) + c.lat12 * F(s1, k, m);
    }
    f3[i + (size_t)ld3 * (k + (size_t)KL * m)] = v;
    fkm = fk; fk = fkp;
  }
}

// Order-preserving float <-> int mapping for atomic max/min of extrema.
__device__ __forceinline__ int f2o(float f) { int i = __float_as_int(f); return i >= 0 ? i : i ^ 0x7fffffff; }
__device__ __forceinline__ long long d2o(double d) { long long i = __double_as_longlong(d); return i >= 0 ? i : i ^ 0x7fffffffffffffffLL; }

// ext[2*c] = max, ext[2*c+1] = min of coefficient class c (CFL_* below)
template <typename R>
__global__ void __launch_bounds__(256) cfl_extrema_kernel(const PropArgs<R> A, long long* ext) {
  const PropCore<R> P(A);
  const size_t n = (size_t)A.nsea * A.KL * A.ML;
  R mx[CFL_NCLASS], mn[CFL_NCLASS];
  for (int c = 0; c < CFL_NCLASS; ++c) { mx[c] = R(-1e30); mn[c] = R(1e30); }
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(t % A.nsea);
    size_t km = t / A.nsea;
    int k = (int)(km % A.KL), m = (int)(km / A.KL);
    Coefs<R> c = P.coef(i, k, m);
    R v[CFL_NCLASS] = {c.lat11, c.lat21, c.lat12, c.lat22, c.lon1, c.lon2, c.th1, c.th2, c.sg1, c.sg2, c.sum};
    for (int q = 0; q < CFL_NCLASS; ++q) { mx[q] = dmax(mx[q], v[q]); mn[q] = dmin(mn[q], v[q]); }
  }
  for (int q = 0; q < CFL_NCLASS; ++q) {
    mx[q] = warp_max(mx[q]);
    R x = mn[q];
    for (int o = 16; o > 0; o >>= 1) x = dmin(x, __shfl_xor_sync(0xffffffffu, x, o));
    mn[q] = x;
  }
  if ((threadIdx.x & 31) == 0)
    for (int q = 0; q < CFL_NCLASS; ++q) {
      long long a = sizeof(R) == 4 ? (long long)f2o((float)mx[q]) : d2o((double)mx[q]);
      long long b = sizeof(R) == 4 ? (long long)f2o((float)mn[q]) : d2o((double)mn[q]);
      atomicMax(&ext[2 * q], a);
      atomicMin(&ext[2 * q + 1], b);
    }
}

__global__ void cfl_init_kernel(long long* ext) {
  int q = threadIdx.x;
  if (q < CFL_NCLASS) { ext[2 * q] = LLONG_MIN; ext[2 * q + 1] = LLONG_MAX; }
}

template <typename R>
cudaError_t launch_propags(const PropArgs<R>& A, const R* f1, int ld1, R* f3, int ld3, cudaStream_t s) {
  if (A.nsea == 0) return cudaSuccess;
  dim3 grid((A.nsea + 127) / 128, A.ML);
  propags_kernel<R><<<grid, 128, 0, s>>>(A, f1, ld1, f3, ld3);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_cfl_extrema(const PropArgs<R>& A, long long* ext, int nsm, cudaStream_t s) {
  cfl_init_kernel<<<1, 32, 0, s>>>(ext);
  size_t n = (size_t)A.nsea * A.KL * A.ML;
  int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)nsm * 8);
  if (blocks < 1) blocks = 1;
  cfl_extrema_kernel<R><<<blocks, 256, 0, s>>>(A, ext);
  return cudaGetLastError();
}

double cfl_decode(long long v, int precision) {
  if (precision == 4) {
    int i = (int)v;
    i = i >= 0 ? i : i ^ 0x7fffffff;
    float f; memcpy(&f, &i, 4); return f;
  }
  long long i = v >= 0 ? v : v ^ 0x7fffffffffffffffLL;
  double d; memcpy(&d, &i, 8); return d;
}

template cudaError_t launch_propags<float>(const PropArgs<float>&, const float*, int, float*, int, cudaStream_t);
template cudaError_t launch_propags<double>(const PropArgs<double>&, const double*, int, double*, int, cudaStream_t);
template cudaError_t launch_cfl_extrema<float>(const PropArgs<float>&, long long*, int, cudaStream_t);
template cudaError_t launch_cfl_extrema<double>(const PropArgs<double>&, long long*, int, cudaStream_t);

}  // namespace wamgpu
