// Integrated output parameters on the device: COMPUTE_OUTPUT_PARAMETER
// (myWAveModel/WAM wam_output_module.f90:481-640) for the parameters that
// are functions of one sea point's spectrum and fields, so that an output
// step reads NSEA x 40 values instead of downloading the spectrum.
//
// One thread integrates one sea point.  The spectrum FL3(IJ,K,M) has the sea
// point fastest, so the 32 threads of a warp read 128 contiguous bytes of
// every bin; the kernel reads the spectrum once (HBM-bound: KL*ML*4 bytes
// per point in, 160 bytes out).  The direction sums of MEAN_DIRECTION and the
// frequency sums of the other integrals are kept per thread in shared memory
// (thread-fastest, conflict-free), and every sum runs in the reference's
// order.  The unit is compiled without FMA contraction, so the results are
// those of the reference's separate operations; only ATAN2 (current
// direction, mean direction) is the device library's.
//
// Routines (wam_interface_module.f90): TOTAL_ENERGY_B :1342-1410, FEMEAN
// :207-286, TM1_TM2_PERIODS_B :1152-1245, PEAK_PERIOD_B :741-813,
// MEAN_DIRECTION_B :412-533, MEANSQS :639-737, CHARNOCK_PAR :159-203; AIRSEA
// (wam_source_module.f90:868-971) when USTAR is zero everywhere.
#include <cfloat>
#include "kernels.hpp"
#include "devmath.cuh"

namespace wamgpu {

namespace {

constexpr int kOutThreads = 128;

template <typename R> struct OutConst {
  static constexpr R DEG = R(180.) / Phys<R>::PI;
};

template <typename R> __device__ __forceinline__ R orient(R deg, int from) {
  return from ? deg : fmod(deg + R(180.), R(360.));
}

// Largest USTAR of the points (non-negative values, ordered as their bit patterns).
template <typename R>
__global__ void __launch_bounds__(256) ustar_max_kernel(const R* __restrict__ ustar, int n, unsigned long long* out) {
  unsigned long long best = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double u = (double)ustar[i];
    if (u > 0) best = max(best, (unsigned long long)__double_as_longlong(u));
  }
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0 && best) atomicMax(out, best);
}

template <typename R>
__global__ void __launch_bounds__(kOutThreads) output_kernel(const __grid_constant__ OutArgs<R> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sm = reinterpret_cast<R*>(smem_raw);
  const int tid = threadIdx.x;
  const int ij = blockIdx.x * kOutThreads + tid;
  if (ij >= a.nsea) return;
  const int kl = a.KL, ml = a.ML;
  using P_ = Phys<R>;
  const R DEG = OutConst<R>::DEG;
  R* Tk = sm + tid;                       // [k * kOutThreads]: direction sums over frequency
  R* Tm = sm + kl * kOutThreads + tid;    // [m * kOutThreads]: frequency spectrum (sum over directions)
  for (int k = 0; k < kl; ++k) Tk[k * kOutThreads] = R(0);
  const R* f = a.fl3 + ij;
  for (int m = 0; m < ml; ++m) {
    const R dfim = a.DFIM[m];
    R s = R(0);
    for (int k = 0; k < kl; ++k) {
      const R v = __ldg(f + (size_t)a.ld * (k + (size_t)kl * m));
      s = s + v;
      Tk[k * kOutThreads] = Tk[k * kOutThreads] + v * dfim;
    }
    Tm[m * kOutThreads] = s;
  }
  R U10 = a.u10[ij], UDIR = a.udir[ij], TAUW = a.tauw[ij];
  R USTAR = a.ustar[ij], Z0 = a.z0[ij];
  if (a.ustar_max && *a.ustar_max == 0ull) {
    // IF (MAXVAL(USTAR(:)).EQ.0.) CALL AIRSEA (U10, TAUW, USTAR, Z0)
    adj::airsea<R, R>(a.A, U10, TAUW, USTAR, Z0);
    a.ustar[ij] = USTAR;
    a.z0[ij] = Z0;
  }
  R* out = a.block + ij;
  auto put = [&](int p, R v) { out[(size_t)a.block_ld * (p - 1)] = v; };
  const R tail = Tm[(ml - 1) * kOutThreads];
  put(1, U10);
  put(2, orient(DEG * UDIR, a.from));
  put(3, USTAR);
  const R TAU = USTAR * USTAR + R(0.0001);
  put(4, TAU / (U10 * U10 + R(0.01)));
  put(16, TAUW / (TAU * P_::ROAIR));
  put(5, P_::G * Z0 / dmax(USTAR * USTAR, R(1.0E-6)));
  put(6, a.shallow ? a.depth[ij] : R(999.));
  const R cu = a.u ? a.u[ij] : R(0), cv = a.v ? a.v[ij] : R(0);
  put(7, sqrt(cu * cu + cv * cv));
  R cdir = orient(atan2(cu, cv) * DEG, a.from);
  if (cdir < R(0.)) cdir = cdir + R(360.);
  put(8, cdir);
  // TOTAL_ENERGY, FEMEAN, TM1, TM2 and MEANSQS: frequency sums in order
  R E = a.MO_TAIL * tail, FM = a.MM1_TAIL * tail, TM1 = a.MP1_TAIL * tail, TM2 = a.MP2_TAIL * tail;
  R SM = R(1.0E-33);  // MAX(CONST2*TEMP(ML), EPSMIN) with CONST2 = 0.*LOG(FC/FS) = 0
  for (int m = 0; m < ml; ++m) {
    const R t = Tm[m * kOutThreads];
    E = E + t * a.DFIM[m];
    FM = FM + t * a.DFIMOFR[m];
    TM1 = TM1 + t * a.DFIM_FR[m];
    TM2 = TM2 + t * a.DFIM_FR2[m];
    if (a.shallow) {
      const R tk = __ldg(&a.TFAK[(a.indep[ij] - 1) + a.NDEPTH * m]);
      SM = SM + a.DFIM[m] * (tk * tk) * t;
    } else {
      SM = SM + a.MSSFD[m] * t;
    }
  }
  E = dmax(E, R(1.0E-12));
  FM = E / dmax(FM, R(1.0E-12));
  put(11, R(1.) / FM);
  put(40, SM);
  put(12, (E > R(1.0E-12)) ? E / TM1 : R(1.));
  put(13, (E > R(1.0E-12)) ? sqrt(E / TM2) : R(1.));
  put(9, R(4.) * sqrt(E));
  // PEAK_PERIOD: the first maximum of the frequency spectrum
  int ip = 0;
  R best = Tm[0];
  for (int m = 1; m < ml; ++m) {
    const R t = Tm[m * kOutThreads];
    if (t > best) { best = t; ip = m; }
  }
  put(10, ip == 0 ? R(1.) : R(1.) / a.FR[ip]);
  // MEAN_DIRECTION: THQ and SPREAD
  R SI = 0, CI = 0, SP = 0;
  for (int k = 0; k < kl; ++k) {
    const R t = Tk[k * kOutThreads];
    SI = SI + a.SINTH[k] * t;
    CI = CI + a.COSTH[k] * t;
    SP = SP + t;
  }
  {
    const R ci = (CI == R(0.)) ? R(0.1E-30) : CI;
    R thq = atan2(SI, ci);
    if (thq < R(0.)) thq = thq + P_::ZPI;
    if (thq > P_::ZPI - R(0.001)) thq = R(0.);
    put(14, orient(thq * DEG, a.from));
  }
  {
    const R lim = R(0.1E-15);
    const R ci = (dabs(CI) < lim) ? copysign(lim, CI) : CI;
    const R si = (dabs(SI) < lim) ? copysign(lim, SI) : SI;
    R sp = (dabs(SP) < lim) ? copysign(lim, SP) : SP;
    sp = R(2.) * (R(1.) - sqrt(si * si + ci * ci) / sp);
    sp = (sp <= R(0)) ? (sizeof(R) == 4 ? R(FLT_MIN) : R(DBL_MIN)) : sqrt(sp);  // TINY(1.)
    put(15, sp * DEG);
  }
  put(32, Z0);
}

}  // namespace

// PUT_ICE / PUT_DRY: rows of the listed sea points set to a value.  One
// thread per (row, listed point): the list is short and scattered, each
// thread writes one element.
template <typename R>
__global__ void __launch_bounds__(256) put_points_kernel(R* __restrict__ data, size_t ld, int nrows,
                                                         const int* __restrict__ points, int n, int lo, int hi, R value) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrows) return;
  const int i = (int)(t % n), row = (int)(t / n);
  const int ij = points[i];  // 1-based sea point number
  if (ij < lo || ij > hi) return;
  data[(size_t)(ij - 1) + ld * row] = value;
}

template <typename R>
cudaError_t launch_put_points(R* data, size_t ld, int nrows, const int* points, int n, int lo, int hi, R value,
                              cudaStream_t s) {
  const size_t total = (size_t)n * nrows;
  if (total == 0) return cudaSuccess;
  put_points_kernel<R><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(data, ld, nrows, points, n, lo, hi, value);
  return cudaGetLastError();
}
template cudaError_t launch_put_points<float>(float*, size_t, int, const int*, int, int, int, float, cudaStream_t);
template cudaError_t launch_put_points<double>(double*, size_t, int, const int*, int, int, int, double, cudaStream_t);

template <typename R> size_t output_smem_bytes(int KL, int ML) { return (size_t)kOutThreads * (KL + ML) * sizeof(R); }

template <typename R> cudaError_t launch_output(const OutArgs<R>& a, unsigned long long* ustar_max, cudaStream_t s) {
  if (a.nsea == 0) return cudaSuccess;
  OutArgs<R> b = a;
  b.ustar_max = nullptr;
  if (ustar_max) {
    cudaError_t e = cudaMemsetAsync(ustar_max, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    ustar_max_kernel<R><<<148, 256, 0, s>>>(a.ustar, a.nsea, ustar_max);
    b.ustar_max = ustar_max;
  }
  const size_t smem = output_smem_bytes<R>(a.KL, a.ML);
  static bool raised[2] = {false, false};
  if (smem > 48 * 1024 && !raised[sizeof(R) == 8]) {
    cudaError_t e = cudaFuncSetAttribute(output_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)output_smem_bytes<R>(MAX_KL, MAX_ML));
    if (e != cudaSuccess) return e;
    raised[sizeof(R) == 8] = true;
  }
  output_kernel<R><<<(a.nsea + kOutThreads - 1) / kOutThreads, kOutThreads, smem, s>>>(b);
  return cudaGetLastError();
}

template cudaError_t launch_output<float>(const OutArgs<float>&, unsigned long long*, cudaStream_t);
template cudaError_t launch_output<double>(const OutArgs<double>&, unsigned long long*, cudaStream_t);
template size_t output_smem_bytes<float>(int, int);
template size_t output_smem_bytes<double>(int, int);

}  // namespace wamgpu
