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

// The integrals COMPUTE_OUTPUT_PARAMETER and SWELL_SEPARATION take of one
// spectrum, from its frequency sums Tm[m * st] (directions summed in order)
// and direction sums Tk[k * st] (DFIM-weighted, frequencies in order):
// TOTAL_ENERGY, FEMEAN, TM1_TM2_PERIODS, PEAK_PERIOD, MEAN_DIRECTION, in the
// statement order of the parameters 9-15 above.
template <typename R> struct SpecInt { R E, TM, TM1, TM2, TP, THQ, SPREAD; };
template <typename R>
__device__ SpecInt<R> spec_integrals(const OutArgs<R>& a, const R* Tk, const R* Tm, int st) {
  using P_ = Phys<R>;
  const int kl = a.KL, ml = a.ML;
  const R DEG = OutConst<R>::DEG;
  SpecInt<R> o;
  const R tail = Tm[(ml - 1) * st];
  R E = a.MO_TAIL * tail, FM = a.MM1_TAIL * tail, TM1 = a.MP1_TAIL * tail, TM2 = a.MP2_TAIL * tail;
  for (int m = 0; m < ml; ++m) {
    const R t = Tm[m * st];
    E = E + t * a.DFIM[m];
    FM = FM + t * a.DFIMOFR[m];
    TM1 = TM1 + t * a.DFIM_FR[m];
    TM2 = TM2 + t * a.DFIM_FR2[m];
  }
  E = dmax(E, R(1.0E-12));
  FM = E / dmax(FM, R(1.0E-12));
  o.E = E;
  o.TM = R(1.) / FM;
  o.TM1 = (E > R(1.0E-12)) ? E / TM1 : R(1.);
  o.TM2 = (E > R(1.0E-12)) ? sqrt(E / TM2) : R(1.);
  int ip = 0;
  R best = Tm[0];
  for (int m = 1; m < ml; ++m) {
    const R t = Tm[m * st];
    if (t > best) { best = t; ip = m; }
  }
  o.TP = ip == 0 ? R(1.) : R(1.) / a.FR[ip];
  R SI = 0, CI = 0, SP = 0;
  for (int k = 0; k < kl; ++k) {
    const R t = Tk[k * st];
    SI = SI + a.SINTH[k] * t;
    CI = CI + a.COSTH[k] * t;
    SP = SP + t;
  }
  {
    const R ci = (CI == R(0.)) ? R(0.1E-30) : CI;
    R thq = atan2(SI, ci);
    if (thq < R(0.)) thq = thq + P_::ZPI;
    if (thq > P_::ZPI - R(0.001)) thq = R(0.);
    o.THQ = orient(thq * DEG, a.from);
  }
  {
    const R lim = R(0.1E-15);
    const R ci = (dabs(CI) < lim) ? copysign(lim, CI) : CI;
    const R si = (dabs(SI) < lim) ? copysign(lim, SI) : SI;
    R sp = (dabs(SP) < lim) ? copysign(lim, SP) : SP;
    sp = R(2.) * (R(1.) - sqrt(si * si + ci * ci) / sp);
    sp = (sp <= R(0)) ? (sizeof(R) == 4 ? R(FLT_MIN) : R(DBL_MIN)) : sqrt(sp);  // TINY(1.)
    o.SPREAD = sp * DEG;
  }
  return o;
}

constexpr int kSwThreads = 64;

// SWELL_SEPARATION (wam_swell_module.f90:106-350) without the partitioning
// (parameters 41-49).  One thread per sea point walks the directions: a bin
// is swell where FRIC/C(M) * 1.2*USTAR*COS(TH(K)-UDIR) < 1, its swell value
// MAX(F, EPSMIN) there and 0 elsewhere, its wind-sea value F minus that.
// The cosine is the correctly rounded single-precision value (the oracle
// forms it the same way, so both split every bin alike).  The frequency sums
// of both spectra still add their directions in order, the direction sums
// their frequencies in order.  Parameters 17-23 (wind sea) and 25-31 (swell):
// Hs, peak period, mean period, TM1, TM2, mean direction, spread.
template <typename R>
__global__ void __launch_bounds__(kSwThreads) swell_kernel(const __grid_constant__ OutArgs<R> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sm = reinterpret_cast<R*>(smem_raw);
  const int tid = threadIdx.x;
  const int ij = blockIdx.x * kSwThreads + tid;
  if (ij >= a.nsea) return;
  const int kl = a.KL, ml = a.ML, st = kSwThreads;
  R* Tk1 = sm + tid;                      // swell direction sums
  R* Tk4 = Tk1 + kl * st;                 // wind-sea direction sums
  R* Tm1 = Tk4 + kl * st;                 // swell frequency sums
  R* Tm4 = Tm1 + ml * st;                 // wind-sea frequency sums
  for (int m = 0; m < ml; ++m) { Tm1[m * st] = R(0); Tm4[m * st] = R(0); }
  const R FRIC = R(28.), EPSMIN = R(0.1E-32);
  const R us = a.ustar[ij], ud = a.udir[ij];
  const R* f = a.fl3 + ij;
  for (int k = 0; k < kl; ++k) {
    const R flpp = R(1.2) * us * crcos(a.TH[k] - ud);
    R t1 = R(0), t4 = R(0);
    for (int m = 0; m < ml; ++m) {
      const R v = __ldg(f + (size_t)a.ld * (k + (size_t)kl * m));
      const R cm = FRIC / a.C[m];
      const R f1 = (cm * flpp < R(1.0)) ? dmax(v, EPSMIN) : R(0.);
      const R f4 = v - f1;
      Tm1[m * st] = Tm1[m * st] + f1;
      Tm4[m * st] = Tm4[m * st] + f4;
      t1 = t1 + f1 * a.DFIM[m];
      t4 = t4 + f4 * a.DFIM[m];
    }
    Tk1[k * st] = t1;
    Tk4[k * st] = t4;
  }
  R* out = a.block + ij;
  auto put = [&](int p, R v) { out[(size_t)a.block_ld * (p - 1)] = v; };
  const SpecInt<R> ws = spec_integrals(a, Tk4, Tm4, st), sw = spec_integrals(a, Tk1, Tm1, st);
  put(17, R(4.) * sqrt(ws.E)); put(18, ws.TP); put(19, ws.TM); put(20, ws.TM1); put(21, ws.TM2);
  put(22, ws.THQ); put(23, ws.SPREAD);
  put(25, R(4.) * sqrt(sw.E)); put(26, sw.TP); put(27, sw.TM); put(28, sw.TM1); put(29, sw.TM2);
  put(30, sw.THQ); put(31, sw.SPREAD);
}

}  // namespace

template <typename R> cudaError_t launch_swell(const OutArgs<R>& a, cudaStream_t s) {
  if (a.nsea == 0) return cudaSuccess;
  const size_t smem = (size_t)kSwThreads * 2 * (a.KL + a.ML) * sizeof(R);
  static bool raised[2] = {false, false};
  if (smem > 48 * 1024 && !raised[sizeof(R) == 8]) {
    cudaError_t e = cudaFuncSetAttribute(swell_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)((size_t)kSwThreads * 2 * (MAX_KL + MAX_ML) * sizeof(R)));
    if (e != cudaSuccess) return e;
    raised[sizeof(R) == 8] = true;
  }
  swell_kernel<R><<<(a.nsea + kSwThreads - 1) / kSwThreads, kSwThreads, smem, s>>>(a);
  return cudaGetLastError();
}
template cudaError_t launch_swell<float>(const OutArgs<float>&, cudaStream_t);
template cudaError_t launch_swell<double>(const OutArgs<double>&, cudaStream_t);

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

// WAM_WIND (wam_wind_module.f90:1063-1216): one input wind field to the sea
// points.  Bilinear interpolation with the tables of INTERPOLATION_TO_GRID
// (:1224-1377; a plain copy on the model's own grid, EQUAL_GRID), then speed
// and direction ATAN2(U,V) in [0, 2*pi), the friction-velocity (CODE_IN 1)
// or surface-stress (2) input turned into U10 through a Charnock drag, and
// U10 >= 2 m/s.  One thread per sea point; the unit rounds every operation
// separately, as the reference does.
template <typename R>
__global__ void __launch_bounds__(256) wind_kernel(const R* __restrict__ u_in, const R* __restrict__ v_in, int nx_in,
                                                   int n, const int* __restrict__ tab, const R* __restrict__ w, int equal,
                                                   int code_in, R* __restrict__ us, R* __restrict__ ds) {
  const int ij = blockIdx.x * blockDim.x + threadIdx.x;
  if (ij >= n) return;
  const int i1 = tab[ij] - 1, i2 = tab[ij + n] - 1, k1 = tab[ij + 2 * n] - 1, k2 = tab[ij + 3 * n] - 1;
  auto at = [&](const R* f, int i, int k) { return __ldg(&f[i + (size_t)nx_in * k]); };
  R uu, vv;
  if (equal) {
    uu = at(u_in, i1, k1);
    vv = at(v_in, i1, k1);
  } else {
    const R di = w[ij], dk = w[ij + n];
    uu = (at(u_in, i1, k1) * (R(1.) - di) + at(u_in, i2, k1) * di) * (R(1.) - dk) +
         (at(u_in, i1, k2) * (R(1.) - di) + at(u_in, i2, k2) * di) * dk;
    vv = (at(v_in, i1, k1) * (R(1.) - di) + at(v_in, i2, k1) * di) * (R(1.) - dk) +
         (at(v_in, i1, k2) * (R(1.) - di) + at(v_in, i2, k2) * di) * dk;
  }
  R s = sqrt(uu * uu + vv * vv);
  R d = (s != R(0.)) ? atan2(uu, vv) : R(0.);
  if (d < R(0.)) d = d + Phys<R>::ZPI;
  if (code_in == 1 || code_in == 2) {
    const R alphach = R(0.0185);
    const R ust = code_in == 1 ? dmax(R(0.01), s) : dmax(R(0.01), sqrt(s / Phys<R>::ROAIR));
    const R z0 = alphach / Phys<R>::G * (ust * ust);
    const R cd = Phys<R>::XKAPPA / log(R(10.) / z0);
    s = ust / cd;
  }
  us[ij] = dmax(s, R(2.0));
  ds[ij] = d;
}

template <typename R>
cudaError_t launch_wind(const R* u_in, const R* v_in, int nx_in, int n, const int* tab, const R* w, int equal,
                        int code_in, R* us, R* ds, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  wind_kernel<R><<<(n + 255) / 256, 256, 0, s>>>(u_in, v_in, nx_in, n, tab, w, equal, code_in, us, ds);
  return cudaGetLastError();
}
template cudaError_t launch_wind<float>(const float*, const float*, int, int, const int*, const float*, int, int, float*,
                                        float*, cudaStream_t);
template cudaError_t launch_wind<double>(const double*, const double*, int, int, const int*, const double*, int, int,
                                         double*, double*, cudaStream_t);

// Restart records: rows b0..b0+nb-1 of a sea-point-fastest device array
// gathered into REAL file order (file position p holds model point perm[p],
// 1-based; perm null = the identity) and scattered back.
template <typename R>
__global__ void __launch_bounds__(256) restart_gather_kernel(const R* __restrict__ src, size_t ld, int nsea,
                                                             const int* __restrict__ perm, int b0, int nb,
                                                             float* __restrict__ out) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)nsea * nb) return;
  const int p = (int)(t % nsea), b = b0 + (int)(t / nsea);
  const int ij = perm ? perm[p] - 1 : p;
  out[t] = (float)src[ij + ld * b];
}
template <typename R>
__global__ void __launch_bounds__(256) restart_scatter_kernel(const float* __restrict__ in, int nsea,
                                                              const int* __restrict__ perm, int b0, int nb,
                                                              R* __restrict__ dst, size_t ld) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)nsea * nb) return;
  const int p = (int)(t % nsea), b = b0 + (int)(t / nsea);
  const int ij = perm ? perm[p] - 1 : p;
  dst[ij + ld * b] = (R)in[t];
}
template <typename R>
cudaError_t launch_restart_gather(const R* src, size_t ld, int nsea, const int* perm, int b0, int nb, float* out,
                                  cudaStream_t s) {
  const size_t n = (size_t)nsea * nb;
  if (n == 0) return cudaSuccess;
  restart_gather_kernel<R><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, ld, nsea, perm, b0, nb, out);
  return cudaGetLastError();
}
template <typename R>
cudaError_t launch_restart_scatter(const float* in, int nsea, const int* perm, int b0, int nb, R* dst, size_t ld,
                                   cudaStream_t s) {
  const size_t n = (size_t)nsea * nb;
  if (n == 0) return cudaSuccess;
  restart_scatter_kernel<R><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, nsea, perm, b0, nb, dst, ld);
  return cudaGetLastError();
}
template cudaError_t launch_restart_gather<float>(const float*, size_t, int, const int*, int, int, float*, cudaStream_t);
template cudaError_t launch_restart_gather<double>(const double*, size_t, int, const int*, int, int, float*, cudaStream_t);
template cudaError_t launch_restart_scatter<float>(const float*, int, const int*, int, int, float*, size_t, cudaStream_t);
template cudaError_t launch_restart_scatter<double>(const float*, int, const int*, int, int, double*, size_t,
                                                    cudaStream_t);

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
