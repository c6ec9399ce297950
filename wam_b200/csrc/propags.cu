// PROPAGS stencil and CHECK_CFL coefficient extrema (compiled with
// -fmad=false so the coefficient arithmetic rounds like the reference).
#include "propags.cuh"
#include "kernels.hpp"

namespace wamgpu {

// One thread per (sea point i, frequency m) walking the directions.
template <typename R, int VAR, bool RED, bool REFRD>
__device__ __forceinline__ void propags_point(const PropArgs<R>& A, const R* __restrict__ f1, int ld1,
                                              R* __restrict__ f3, int ld3, int i, int m) {
  using S = Site<R, VAR, RED, REFRD>;
  const S site(A, i, m);
  const int KL = A.KL, ML = A.ML;
  const size_t plane = (size_t)ld1 * KL;
  const R* fm = f1 + plane * m;
  auto F = [&](int p1, int k) -> R { return p1 == 0 ? R(0) : __ldg(&fm[(p1 - 1) + (size_t)ld1 * k]); };
  const bool theta = REFRD || S::SPH;
  R fkm = F(i + 1, KL - 1), fk = F(i + 1, 0);
  R* out = f3 + i + (size_t)ld3 * KL * m;
  typename S::Win W = site.window(0);
  for (int k = 0; k < KL; ++k) {
    const int kp = (k + 1 == KL) ? 0 : k + 1;
    const R fkp = F(i + 1, kp);
    const Coefs<R> c = site.coef_w(W);
    R v;
    if (!S::CUR) {
      const bool ic0 = W.cs >= R(0.), is0 = W.sn >= R(0.);
      v = c.sum * fk + c.lat11 * F(ic0 ? site.s0 : site.n0, k) + c.lon1 * F(is0 ? site.w0 : site.e0, k);
      if (theta) v = v + c.th1 * fkp + c.th2 * fkm;
      if (RED) v = v + c.lat12 * F(ic0 ? site.s1 : site.n1, k);
    } else {
      const int mm = (m == 0) ? 0 : m - 1, mp = (m == ML - 1) ? ML - 1 : m + 1;
      const R fmp = __ldg(&f1[i + (size_t)ld1 * k + plane * mp]), fmm = __ldg(&f1[i + (size_t)ld1 * k + plane * mm]);
      v = c.sum * fk + c.lat21 * F(site.n0, k) + c.lat11 * F(site.s0, k) + c.lon2 * F(site.e0, k) +
          c.lon1 * F(site.w0, k) + c.th1 * fkp + c.th2 * fkm + c.sg1 * fmp + c.sg2 * fmm;
      if (RED) v = v + c.lat22 * F(site.n1, k) + c.lat12 * F(site.s1, k);
    }
    out[(size_t)ld3 * k] = v;
    fkm = fk; fk = fkp;
    site.advance(W, k);
  }
}

template <typename R, int VAR, bool RED, bool REFRD>
__global__ void __launch_bounds__(128) propags_kernel(const __grid_constant__ PropArgs<R> A, const R* __restrict__ f1,
                                                      int ld1, R* __restrict__ f3, int ld3, int m0) {
  const int i = A.i0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.i1) return;
  propags_point<R, VAR, RED, REFRD>(A, f1, ld1, f3, ld3, i, m0 + blockIdx.y);
}

// Two frequencies m, m+1 of one sea point per thread, for the variants
// without currents (a sub-step of plane m then reads plane m only).  The
// direction-dependent work that does not depend on the frequency (direction
// tables, upwind neighbour choice and addresses, |SIN|, |COS| and the metric
// products, the depth-gradient part of THDD) is the same expression for both
// frequencies and is formed once; every coefficient still gets the
// reference's operations, so the result equals the one-frequency kernel's.
// With mb beyond the planes (odd count) the second frequency repeats the
// first and is not stored.
template <typename R, int VAR, bool RED, bool REFRD>
__device__ __forceinline__ void propags_point2(const PropArgs<R>& A, const R* __restrict__ f1, int ld1,
                                               R* __restrict__ f3, int ld3, int i, int m, bool two) {
  using S = Site<R, VAR, RED, REFRD>;
  static_assert(!S::CUR, "two-frequency PROPAGS is for the variants without currents");
  const int mb = two ? m + 1 : m;
  const S sa(A, i, m), sb(A, i, mb);
  const int KL = A.KL;
  const size_t plane = (size_t)ld1 * KL;
  const R* fa = f1 + plane * m;
  const R* fb = f1 + plane * mb;
  const bool theta = REFRD || S::SPH;
  auto at = [&](const R* fm, int p1, int k) -> R { return p1 == 0 ? R(0) : __ldg(&fm[(p1 - 1) + (size_t)ld1 * k]); };
  R fkm_a = at(fa, i + 1, KL - 1), fk_a = at(fa, i + 1, 0);
  R fkm_b = at(fb, i + 1, KL - 1), fk_b = at(fb, i + 1, 0);
  R* outa = f3 + i + (size_t)ld3 * KL * m;
  R* outb = f3 + i + (size_t)ld3 * KL * mb;
  typename S::Win Wa = sa.window(0), Wb = sb.window(0);
  for (int k = 0; k < KL; ++k) {
    const int kp = (k + 1 == KL) ? 0 : k + 1;
    const R fkp_a = at(fa, i + 1, kp), fkp_b = at(fb, i + 1, kp);
    const Coefs<R> ca = sa.coef_w(Wa), cb = sb.coef_w(Wb);
    const bool ic0 = Wa.cs >= R(0.), is0 = Wa.sn >= R(0.);
    const int pl = ic0 ? sa.s0 : sa.n0, pw = is0 ? sa.w0 : sa.e0;
    R va = ca.sum * fk_a + ca.lat11 * at(fa, pl, k) + ca.lon1 * at(fa, pw, k);
    R vb = cb.sum * fk_b + cb.lat11 * at(fb, pl, k) + cb.lon1 * at(fb, pw, k);
    if (theta) { va = va + ca.th1 * fkp_a + ca.th2 * fkm_a; vb = vb + cb.th1 * fkp_b + cb.th2 * fkm_b; }
    if (RED) {
      const int p2 = ic0 ? sa.s1 : sa.n1;
      va = va + ca.lat12 * at(fa, p2, k);
      vb = vb + cb.lat12 * at(fb, p2, k);
    }
    outa[(size_t)ld3 * k] = va;
    if (two) outb[(size_t)ld3 * k] = vb;
    fkm_a = fk_a; fk_a = fkp_a; fkm_b = fk_b; fk_b = fkp_b;
    sa.advance(Wa, k);
    sb.advance(Wb, k);
  }
}

// Frequencies m0 + 2*blockIdx.y and the next one (if below m0 + mcount).
template <typename R, int VAR, bool RED, bool REFRD>
__global__ void __launch_bounds__(128) propags2_kernel(const __grid_constant__ PropArgs<R> A, const R* __restrict__ f1,
                                                       int ld1, R* __restrict__ f3, int ld3, int m0, int mcount) {
  const int i = A.i0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.i1) return;
  const int q = 2 * blockIdx.y;
  propags_point2<R, VAR, RED, REFRD>(A, f1, ld1, f3, ld3, i, m0 + q, q + 1 < mcount);
}

// Batched form: every member of an ensemble (one coefficient family) in one
// launch of BS-point CTAs.  CTA b belongs to member g with first[g] <= b <
// first[g + 1] and covers frequency m and points ib*BS .. of that member; the
// member's metadata block (direction tables included) is copied into shared
// memory first.
template <typename R, int VAR, bool RED, bool REFRD, int BS>
__global__ void __launch_bounds__(BS) propags_batch_kernel(const PropMember<R>* __restrict__ mem,
                                                           const int* __restrict__ first, int nmem) {
  __shared__ __align__(16) PropMember<R> sm;
  __shared__ int sg;
  if (threadIdx.x == 0) {
    int lo = 0, hi = nmem - 1;
    while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (first[mid] <= (int)blockIdx.x) lo = mid; else hi = mid - 1; }
    sg = lo;
  }
  __syncthreads();
  const int g = sg;
  {
    const int nw = (int)(sizeof(PropMember<R>) / sizeof(int));
    const int* src = reinterpret_cast<const int*>(mem + g);
    int* dst = reinterpret_cast<int*>(&sm);
    for (int q = threadIdx.x; q < nw; q += BS) dst[q] = src[q];
  }
  __syncthreads();
  const int lb = (int)blockIdx.x - first[g], m = lb / sm.nbi, ib = lb - m * sm.nbi;
  const int i = sm.A.i0 + ib * BS + threadIdx.x;
  if (i >= sm.A.i1) return;
  propags_point<R, VAR, RED, REFRD>(sm.A, sm.src, sm.ld, sm.dst, sm.ld, i, m);
}

// Transpose of one sub-step, thread per (sea point i, frequency m): every
// term c * F_old(source) of the forward stencil becomes lam_old(source) +=
// c * lam_new(i, k, m).  The own point's direction neighbours (refraction)
// and the point itself are summed in registers first; spatial and frequency
// neighbours take atomic adds (lam_old zeroed by the caller).
template <typename R, int VAR, bool RED, bool REFRD>
__global__ void __launch_bounds__(128) propags_adj_kernel(const __grid_constant__ PropArgs<R> A,
                                                          const R* __restrict__ lnew, int ld1, R* lold, int ld3) {
  const int i = A.i0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.i1) return;
  const int m = blockIdx.y;
  using S = Site<R, VAR, RED, REFRD>;
  const S site(A, i, m);
  const int KL = A.KL, ML = A.ML;
  const size_t plane = (size_t)ld3 * KL;
  const R* lm = lnew + (size_t)ld1 * KL * m;
  R* om = lold + plane * m;
  auto add = [&](int p1, int k, R v) { if (p1 != 0) atomicAdd(&om[(p1 - 1) + (size_t)ld3 * k], v); };
  const bool theta = REFRD || S::SPH;
  typename S::Win W = site.window(0);
  R carry0 = 0, first_th2 = 0, prev_own = 0;  // own-point sums waiting for the next direction
  for (int k = 0; k < KL; ++k) {
    const Coefs<R> c = site.coef_w(W);
    const R l = lm[i + (size_t)ld1 * k];
    R own = c.sum * l + carry0;  // + th1 of direction k-1 (carried)
    carry0 = 0;
    if (!S::CUR) {
      const bool ic0 = W.cs >= R(0.), is0 = W.sn >= R(0.);
      add(ic0 ? site.s0 : site.n0, k, c.lat11 * l);
      add(is0 ? site.w0 : site.e0, k, c.lon1 * l);
      if (RED) add(ic0 ? site.s1 : site.n1, k, c.lat12 * l);
    } else {
      add(site.n0, k, c.lat21 * l); add(site.s0, k, c.lat11 * l); add(site.e0, k, c.lon2 * l); add(site.w0, k, c.lon1 * l);
      if (RED) { add(site.n1, k, c.lat22 * l); add(site.s1, k, c.lat12 * l); }
      const int mm = (m == 0) ? 0 : m - 1, mp = (m == ML - 1) ? ML - 1 : m + 1;
      atomicAdd(&lold[i + (size_t)ld3 * k + plane * mp], c.sg1 * l);
      atomicAdd(&lold[i + (size_t)ld3 * k + plane * mm], c.sg2 * l);
    }
    if (theta || S::CUR) {
      // F_new(k) reads F_old(k+1) with th1 and F_old(k-1) with th2
      carry0 = c.th1 * l;                 // -> direction k+1
      if (k == 0) first_th2 = c.th2 * l;  // -> direction KL-1, added at the end
      else prev_own = prev_own + c.th2 * l;
    }
    if (k > 0) atomicAdd(&om[i + (size_t)ld3 * (k - 1)], prev_own);
    prev_own = own;
    site.advance(W, k);
  }
  // direction KL-1 gets its own sum and th2 of direction 0; direction 0 gets th1 of KL-1
  atomicAdd(&om[i + (size_t)ld3 * (KL - 1)], prev_own + first_th2);
  if (theta || S::CUR) atomicAdd(&om[i], carry0);
}

// Order-preserving float <-> int mapping for atomic max/min of extrema.
__device__ __forceinline__ int f2o(float f) { int i = __float_as_int(f); return i >= 0 ? i : i ^ 0x7fffffff; }
__device__ __forceinline__ long long d2o(double d) { long long i = __double_as_longlong(d); return i >= 0 ? i : i ^ 0x7fffffffffffffffLL; }

// ext[2*c] = max, ext[2*c+1] = min of coefficient class c (CflClass)
template <typename R, int VAR, bool RED, bool REFRD>
__global__ void __launch_bounds__(256) cfl_extrema_kernel(const __grid_constant__ PropArgs<R> A, long long* ext) {
  const int nown = A.i1 - A.i0;
  const size_t n = (size_t)nown * A.ML;
  R mx[CFL_NCLASS], mn[CFL_NCLASS];
  for (int c = 0; c < CFL_NCLASS; ++c) { mx[c] = R(-1e30); mn[c] = R(1e30); }
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int i = A.i0 + (int)(t % nown), m = (int)(t / nown);
    const Site<R, VAR, RED, REFRD> site(A, i, m);
    for (int k = 0; k < A.KL; ++k) {
      Coefs<R> c = site.coef(k);
      R v[CFL_NCLASS] = {c.lat11, c.lat21, c.lat12, c.lat22, c.lon1, c.lon2, c.th1, c.th2, c.sg1, c.sg2, c.sum};
      for (int q = 0; q < CFL_NCLASS; ++q) { mx[q] = dmax(mx[q], v[q]); mn[q] = dmin(mn[q], v[q]); }
    }
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

// Compile-time dispatch over the ten reference variants (eight coefficient
// families x reduced grid x depth refraction).
template <typename R, template <typename, int, bool, bool> class K, typename... Args>
cudaError_t dispatch(const PropArgs<R>& A, Args&&... args) {
  const bool red = A.reduced != 0, rd = A.refr_d != 0;
#define VCASE(V)                                                             \
  case V:                                                                    \
    if (red) { if (rd) return K<R, V, true, true>::run(A, args...); return K<R, V, true, false>::run(A, args...); } \
    if (rd) return K<R, V, false, true>::run(A, args...);                    \
    return K<R, V, false, false>::run(A, args...);
  switch (A.variant) {
    VCASE(V_CART_DEEP) VCASE(V_CART_SHALLOW) VCASE(V_CART_DEEP_CUR) VCASE(V_CART_SHALLOW_CUR)
    VCASE(V_SPHER_DEEP) VCASE(V_SPHER_SHALLOW) VCASE(V_SPHER_DEEP_CURR) VCASE(V_SPHER_SHALLOW_CURR)
  }
#undef VCASE
  return cudaErrorInvalidValue;
}

template <typename R, int V, bool RED, bool RD> struct PropLaunch {
  static cudaError_t run(const PropArgs<R>& A, const R* f1, int ld1, R* f3, int ld3, int m0, int mcount, cudaStream_t s) {
    if constexpr (!var_current(V)) {
      if (mcount >= 2) {
        dim3 grid((A.i1 - A.i0 + 127) / 128, (mcount + 1) / 2);
        propags2_kernel<R, V, RED, RD><<<grid, 128, 0, s>>>(A, f1, ld1, f3, ld3, m0, mcount);
        return cudaGetLastError();
      }
    }
    dim3 grid((A.i1 - A.i0 + 127) / 128, mcount);
    propags_kernel<R, V, RED, RD><<<grid, 128, 0, s>>>(A, f1, ld1, f3, ld3, m0);
    return cudaGetLastError();
  }
};
template <typename R, int V, bool RED, bool RD> struct CflLaunch {
  static cudaError_t run(const PropArgs<R>& A, long long* ext, int blocks, cudaStream_t s) {
    cfl_extrema_kernel<R, V, RED, RD><<<blocks, 256, 0, s>>>(A, ext);
    return cudaGetLastError();
  }
};

template <typename R, int V, bool RED, bool RD> struct PropBatchLaunch {
  static cudaError_t run(const PropArgs<R>&, const PropMember<R>* mem, const int* first, int nmem, int nblocks, int bs,
                         cudaStream_t s) {
    if (bs == 128) propags_batch_kernel<R, V, RED, RD, 128><<<nblocks, 128, 0, s>>>(mem, first, nmem);
    else if (bs == 256) propags_batch_kernel<R, V, RED, RD, 256><<<nblocks, 256, 0, s>>>(mem, first, nmem);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
  }
};

template <typename R>
cudaError_t launch_propags_batch(const PropArgs<R>& family, const PropMember<R>* mem, const int* first, int nmem,
                                 int nblocks, int bs, cudaStream_t s) {
  if (nblocks == 0) return cudaSuccess;
  return dispatch<R, PropBatchLaunch>(family, mem, first, nmem, nblocks, bs, s);
}

template <typename R, int V, bool RED, bool RD> struct PropAdjLaunch {
  static cudaError_t run(const PropArgs<R>& A, const R* ln, int ld1, R* lo, int ld3, cudaStream_t s) {
    dim3 grid((A.i1 - A.i0 + 127) / 128, A.ML);
    propags_adj_kernel<R, V, RED, RD><<<grid, 128, 0, s>>>(A, ln, ld1, lo, ld3);
    return cudaGetLastError();
  }
};

template <typename R>
cudaError_t launch_propags_adj(const PropArgs<R>& A, const R* lam_new, int ld1, R* lam_old, int ld3, cudaStream_t s) {
  if (A.i1 <= A.i0) return cudaSuccess;
  return dispatch<R, PropAdjLaunch>(A, lam_new, ld1, lam_old, ld3, s);
}

template <typename R>
cudaError_t launch_propags(const PropArgs<R>& A, const R* f1, int ld1, R* f3, int ld3, cudaStream_t s, int m0, int mcount) {
  if (mcount < 0) mcount = A.ML - m0;
  if (m0 < 0 || mcount < 0 || m0 + mcount > A.ML) return cudaErrorInvalidValue;
  if (A.i1 <= A.i0 || mcount == 0) return cudaSuccess;
  return dispatch<R, PropLaunch>(A, f1, ld1, f3, ld3, m0, mcount, s);
}

bool propags_planes_independent(int variant) {
  return variant != V_CART_DEEP_CUR && variant != V_CART_SHALLOW_CUR && variant != V_SPHER_DEEP_CURR &&
         variant != V_SPHER_SHALLOW_CURR;
}

template <typename R>
cudaError_t launch_cfl_extrema(const PropArgs<R>& A, long long* ext, int nsm, cudaStream_t s) {
  cfl_init_kernel<<<1, 32, 0, s>>>(ext);
  if (A.i1 <= A.i0) return cudaGetLastError();
  size_t n = (size_t)(A.i1 - A.i0) * A.ML;
  int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)nsm * 8);
  if (blocks < 1) blocks = 1;
  return dispatch<R, CflLaunch>(A, ext, blocks, s);
}

// Fixed F1 ping-pong spectrum of wamgpu_propags_dev_static: one per device,
// reserved when the module loads, never allocated or freed by the library.
static __device__ __align__(256) unsigned char g_static_prop_scratch[WAMGPU_STATIC_SCRATCH_BYTES];

// Device address of g_static_prop_scratch on the current device.
cudaError_t static_scratch_address(void** p) { return cudaGetSymbolAddress(p, g_static_prop_scratch); }

double cfl_decode(long long v, int precision) {
  if (precision == 4) {
    int i = (int)v;
    i = i >= 0 ? i : i ^ 0x7fffffff;
    float f; memcpy(&f, &i, 4); return f;
  }
  long long i = v >= 0 ? v : v ^ 0x7fffffffffffffffLL;
  double d; memcpy(&d, &i, 8); return d;
}

template cudaError_t launch_propags<float>(const PropArgs<float>&, const float*, int, float*, int, cudaStream_t, int, int);
template cudaError_t launch_propags<double>(const PropArgs<double>&, const double*, int, double*, int, cudaStream_t, int, int);
template cudaError_t launch_propags_batch<float>(const PropArgs<float>&, const PropMember<float>*, const int*, int, int,
                                                 int, cudaStream_t);
template cudaError_t launch_propags_batch<double>(const PropArgs<double>&, const PropMember<double>*, const int*, int,
                                                  int, int, cudaStream_t);
template cudaError_t launch_propags_adj<float>(const PropArgs<float>&, const float*, int, float*, int, cudaStream_t);
template cudaError_t launch_propags_adj<double>(const PropArgs<double>&, const double*, int, double*, int, cudaStream_t);
template cudaError_t launch_cfl_extrema<float>(const PropArgs<float>&, long long*, int, cudaStream_t);
template cudaError_t launch_cfl_extrema<double>(const PropArgs<double>&, long long*, int, cudaStream_t);

}  // namespace wamgpu
