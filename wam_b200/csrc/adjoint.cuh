// Point-per-thread restatement of IMPLSCH for ST4 (IPHYS=1), templated on
// the number type, for the tangent-linear model and the scalar routines the
// adjoint differentiates.
//
//  - `forward<R,T>` restates IMPLSCH (wam_source_module.f90:374-700, the ST4
//    branches) statement by statement for one sea point, its per-point
//    arrays in global memory with the sea point fastest ([bin * ld + ij]) so
//    that the 32 threads of a warp touch 32 consecutive addresses.  T = R
//    gives the values (with a tape of intermediates); T = Dual<R> gives the
//    tangent-linear model: the value and the directional derivative of every
//    statement.
//  - The scalar routines with two inputs (AIRSEA's Newton iteration,
//    TAU_PHI_HF, WSIGSTAR) are written once for any T, so the adjoint kernel
//    (adjoint_warp.cuh) differentiates them by two dual-number passes, which
//    is exact for the computation as done.
//
// Discrete decisions (the cut-off index MIJ, the wind-sea mask LLWS, JU,
// branches of MAX/MIN and the limiter) are those of the forward state and are
// held fixed, as a linearisation of the computed function does.
#pragma once
#include <cfloat>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include "spectral_tables.hpp"

#if defined(__CUDACC__)
#define WAHD __host__ __device__ __forceinline__
#else
#define WAHD inline
#endif

namespace wamgpu {
namespace adj {

// ---- numbers ------------------------------------------------------------------

template <typename R> struct Dual {
  R v, d;
  WAHD Dual() : v(0), d(0) {}
  WAHD Dual(R x) : v(x), d(0) {}
  WAHD Dual(R x, R dx) : v(x), d(dx) {}
};
template <typename T> struct Base { using type = T; };
template <typename R> struct Base<Dual<R>> { using type = R; };

WAHD float val(float x) { return x; }
WAHD double val(double x) { return x; }
template <typename R> WAHD R val(const Dual<R>& x) { return x.v; }

template <typename R> WAHD Dual<R> operator+(Dual<R> a, Dual<R> b) { return Dual<R>(a.v + b.v, a.d + b.d); }
template <typename R> WAHD Dual<R> operator-(Dual<R> a, Dual<R> b) { return Dual<R>(a.v - b.v, a.d - b.d); }
template <typename R> WAHD Dual<R> operator*(Dual<R> a, Dual<R> b) { return Dual<R>(a.v * b.v, a.d * b.v + a.v * b.d); }
template <typename R> WAHD Dual<R> operator/(Dual<R> a, Dual<R> b) {
  const R q = a.v / b.v;
  return Dual<R>(q, (a.d - q * b.d) / b.v);
}
template <typename R> WAHD Dual<R> operator-(Dual<R> a) { return Dual<R>(-a.v, -a.d); }
#define WA_MIXED(OP)                                                                                  \
  template <typename R> WAHD Dual<R> operator OP(Dual<R> a, R b) { return a OP Dual<R>(b); }          \
  template <typename R> WAHD Dual<R> operator OP(R a, Dual<R> b) { return Dual<R>(a) OP b; }
WA_MIXED(+) WA_MIXED(-) WA_MIXED(*) WA_MIXED(/)
#undef WA_MIXED
#define WA_CMP(OP)                                                                                    \
  template <typename R> WAHD bool operator OP(Dual<R> a, Dual<R> b) { return a.v OP b.v; }            \
  template <typename R> WAHD bool operator OP(Dual<R> a, R b) { return a.v OP b; }                    \
  template <typename R> WAHD bool operator OP(R a, Dual<R> b) { return a OP b.v; }
WA_CMP(<) WA_CMP(>) WA_CMP(<=) WA_CMP(>=) WA_CMP(==) WA_CMP(!=)
#undef WA_CMP

WAHD float mexp(float x) { return expf(x); }
WAHD double mexp(double x) { return exp(x); }
WAHD float mlog(float x) { return logf(x); }
WAHD double mlog(double x) { return log(x); }
WAHD float mlog10(float x) { return log10f(x); }
WAHD double mlog10(double x) { return log10(x); }
WAHD float msqrt(float x) { return sqrtf(x); }
WAHD double msqrt(double x) { return sqrt(x); }
WAHD float mpow(float x, float y) { return powf(x, y); }
WAHD double mpow(double x, double y) { return pow(x, y); }
WAHD float mtanh(float x) { return tanhf(x); }
WAHD double mtanh(double x) { return tanh(x); }
WAHD float mcos(float x) { return cosf(x); }
WAHD double mcos(double x) { return cos(x); }
WAHD float msin(float x) { return sinf(x); }
WAHD double msin(double x) { return sin(x); }
WAHD float matan2(float y, float x) { return atan2f(y, x); }
WAHD double matan2(double y, double x) { return atan2(y, x); }
WAHD float mabs(float x) { return fabsf(x); }
WAHD double mabs(double x) { return fabs(x); }
WAHD float msinh(float x) { return sinhf(x); }
WAHD double msinh(double x) { return sinh(x); }

template <typename R> WAHD Dual<R> mexp(Dual<R> a) { const R e = mexp(a.v); return Dual<R>(e, e * a.d); }
template <typename R> WAHD Dual<R> mlog(Dual<R> a) { return Dual<R>(mlog(a.v), a.d / a.v); }
template <typename R> WAHD Dual<R> mlog10(Dual<R> a) { return Dual<R>(mlog10(a.v), a.d / (a.v * mlog(R(10)))); }
template <typename R> WAHD Dual<R> msqrt(Dual<R> a) { const R s = msqrt(a.v); return Dual<R>(s, s > R(0) ? a.d / (R(2) * s) : R(0)); }
template <typename R> WAHD Dual<R> mpow(Dual<R> a, R y) {
  const R p = mpow(a.v, y);
  return Dual<R>(p, a.v != R(0) ? y * p / a.v * a.d : R(0));
}
template <typename R> WAHD Dual<R> mtanh(Dual<R> a) { const R t = mtanh(a.v); return Dual<R>(t, (R(1) - t * t) * a.d); }
template <typename R> WAHD Dual<R> mcos(Dual<R> a) { return Dual<R>(mcos(a.v), -msin(a.v) * a.d); }
template <typename R> WAHD Dual<R> msin(Dual<R> a) { return Dual<R>(msin(a.v), mcos(a.v) * a.d); }
template <typename R> WAHD Dual<R> matan2(Dual<R> y, Dual<R> x) {
  const R q = x.v * x.v + y.v * y.v;
  return Dual<R>(matan2(y.v, x.v), q > R(0) ? (x.v * y.d - y.v * x.d) / q : R(0));
}
template <typename R> WAHD Dual<R> mabs(Dual<R> a) { return a.v < R(0) ? -a : a; }
// Fortran MAX/MIN on ordered operands (the forward kernel's dmax/dmin): the
// selected operand carries its derivative
template <typename A, typename B> WAHD auto mmax(A a, B b) -> decltype(a + b) {
  using C = decltype(a + b);
  return a < b ? C(b) : C(a);
}
template <typename A, typename B> WAHD auto mmin(A a, B b) -> decltype(a + b) {
  using C = decltype(a + b);
  return b < a ? C(b) : C(a);
}

// ---- tables and per-point data -------------------------------------------------

// Static source tables of one spectral grid (the forward kernel's tables).
template <typename R> struct ATabs {
  int KL, ML, NDEPTH, MFRSTLW, MLSTHG, KFRH, NSDSNTH, shallow, isnonlin;
  R DELTH, INV_LOG_CO, MO_TAIL, MM1_TAIL, DELU, DAL1, DAL2, X0TAUHF, BETAMAX, ZALP, ALPHA, TAUWSHELTER, DELT;
  const R *FR, *DFIM, *DFIMOFR, *FR5, *FRM5, *RHOWG, *TH, *COSTH, *SINTH, *DELFL, *AF11, *RNL, *SATW, *WTAUHF, *SWELLFT;
  const R *TFAK, *TCGOND, *FLMINFR;
  const int *K1W, *K2W, *K11W, *K21W, *INL, *IKP, *IKP1, *IKM, *IKM1, *INDSAT;
};

// One column of a per-point array: element b at p[b * ld].
template <typename X> struct Col {
  X* p;
  size_t ld;
  WAHD X& operator[](int b) const { return p[(size_t)b * ld]; }
};

// Inputs of one point that are not differentiated.
template <typename R> struct PointIn {
  int INDEP;
  R DEPTH, UDIR, ROAIRN, WSTAR;
  Col<const R> ENH;  // MAKE_SHALLOW_SNL factors per MC (ISNONLIN != 0), else p == null
};

// Tape layout (per point, in elements of T): for each SINPUT_ARD call c = 0, 1
// the sheltering sums entering every frequency (xst, yst of the two gust
// branches) and the per-frequency SPOS sums ST, SX, SY; then scalars.
WAHD int tape_sin(int c, int q, int ML) { return (7 * c + q) * ML; }  // q: 0,1 xst; 2,3 yst; 4 ST; 5 SX; 6 SY
enum TapeScalar { TS_USTAR1, TS_Z01, TS_TAUW1, TS_USTAR2, TS_Z02, TS_TAUW2, TS_EMEAN, TS_FMEAN, TS_AKMEAN, TS_EMEANWS,
                  TS_FMEANWS, TS_COUNT };
WAHD int tape_scalar(int q, int ML) { return 14 * ML + q; }
WAHD int tape_size(int ML) { return 14 * ML + TS_COUNT; }
// Integer tape: MIJ, MIJ after the update, JU.
enum TapeInt { TI_MIJ, TI_MIJ2, TI_JU, TI_COUNT };

template <typename R> WAHD R tfak(const ATabs<R>& A, const PointIn<R>& P, int m) { return A.TFAK[(P.INDEP - 1) + A.NDEPTH * m]; }
template <typename R> WAHD R tcgond(const ATabs<R>& A, const PointIn<R>& P, int m) { return A.TCGOND[(P.INDEP - 1) + A.NDEPTH * m]; }


// ---- forward routines (ST4), statement order of the forward kernel ------------

// TOTAL_ENERGY + FEMEAN (+ WM1 for AKMEAN), masked by LLWS when mask.p != null
// (wam_interface_module.f90:1342,207,1591).
template <typename R, typename T, typename FC>
WAHD void integrals(const ATabs<R>& A, const PointIn<R>& P, FC F, Col<const uint8_t> mask, T& emean, T& fmean,
                    T* akmean) {
  using Ph = Phys<R>;
  const int kl = A.KL, ml = A.ML;
  T pe = R(0), pf = R(0), pa = R(0), tail = R(0);
  const R DEL2 = msqrt(Ph::G) / Ph::ZPI;
  for (int m = 0; m < ml; ++m) {
    T t = R(0);
    for (int k = 0; k < kl; ++k) {
      const int b = k + kl * m;
      if (!mask.p || mask[b]) t = t + F[b];
    }
    pe = pe + t * A.DFIM[m];
    pf = pf + t * A.DFIMOFR[m];
    if (akmean) pa = pa + (A.shallow ? t / msqrt(tfak(A, P, m)) * A.DFIM[m] : t * A.DFIMOFR[m] * DEL2);
    if (m == ml - 1) tail = t;
  }
  emean = mmax(A.MO_TAIL * tail + pe, R(1.0E-12));
  fmean = emean / mmax(A.MM1_TAIL * tail + pf, R(1.0E-12));
  if (akmean) {
    T wm = A.MM1_TAIL * DEL2 * tail + pa;
    *akmean = (emean > R(1.0E-12)) ? (emean / wm) * (emean / wm) : T(R(1.));
  }
}

// AIRSEA (wam_source_module.f90:868-971): u* and z0 from U10 and the wave stress.
template <typename R, typename T>
WAHD void airsea(const ATabs<R>& A, T U10, T TAUW, T& USTAR, T& Z0) {
  using Ph = Phys<R>;
  const R EPS1 = R(0.00001);
  const R xlogxl = mlog(Ph::XNLEV), alphaog = A.ALPHA / Ph::G;
  T xkutop = Ph::XKAPPA * U10;
  T ustold = U10 * msqrt(R(8.0E-4) + R(8.0E-5) * U10);
  T tauold = mmax(ustold * ustold, TAUW + EPS1);
  USTAR = msqrt(tauold);
  T ustm1 = R(1.0) / mmax(USTAR, R(1.0E-6));
  T z0ch = R(0);
  for (int it = 0; it < 15; ++it) {
    T x = TAUW / tauold;
    z0ch = alphaog * tauold / msqrt(mmax(R(1.0) - x, EPS1));
    T z0vis = Ph::RNUAIRM * ustm1, z0tot = z0ch + z0vis;
    T xologz0 = R(1.0) / (xlogxl - mlog(z0tot));
    T f = USTAR - xkutop * xologz0;
    T zz = ustm1 * (z0ch * (R(2.0) - R(3.0) * x) / (R(1.0) - x) - z0vis) / z0tot;
    T delf = R(1.0) - xkutop * (xologz0 * xologz0) * zz;
    USTAR = USTAR - f / delf;
    T taunew = mmax(USTAR * USTAR, TAUW + EPS1);
    USTAR = msqrt(taunew);
    if (taunew == tauold) break;
    ustm1 = R(1.0) / mmax(USTAR, R(1.0E-6));
    tauold = taunew;
  }
  Z0 = z0ch;
}

// WSIGSTAR (:4250-4339): gustiness from the convective velocity WSTAR.
template <typename R, typename T>
WAHD T wsigstar(const PointIn<R>& P, T ustar, T z0) {
  using Ph = Phys<R>;
  const R C1 = R(1.03E-3), C2 = R(0.04E-3), P1 = R(1.48), P2 = R(-0.21);
  T u = ustar * (R(1.0) / Ph::XKAPPA) * (mlog(R(10.0)) - mlog(z0));
  u = mmax(u, R(1.0));
  T um1 = R(1.0) / u, c2u = C2 * mpow(u, P1), up2 = mpow(u, P2);
  T cdv = (C1 + c2u) * up2;
  T dcd = (P2 * C1 + (P1 + P2) * c2u) * up2 * um1;
  T sconv = R(1.0) + R(0.5) * u / cdv * dcd;
  return mmin(R(0.1), sconv * um1 * mpow(R(0.5) * Ph::XKAPPA * (P.WSTAR * P.WSTAR * P.WSTAR), R(1.0) / R(3.0)));
}

// Constants of SINPUT_ARD (:2312-2738).
template <typename R> struct SinK {
  static constexpr R SWELLF = R(0.66), FU = R(0.022), FUD = R(-0.018), SWELLF4 = R(1.5E05), SWELLF5 = R(1.2),
                     SWELLF7 = R(3.6E05);
};

// SINPUT_ARD: SL, FL, LLWS per bin and the per-frequency SPOS sums (tape);
// records the sheltering sums entering each frequency (tape).
template <typename R, typename T, typename FC>
WAHD void sinput(const ATabs<R>& A, const PointIn<R>& P, FC F, T USTAR, T Z0, Col<T> SL, Col<T> FL, Col<uint8_t> LL,
                 Col<T> tape, int call) {
  using Ph = Phys<R>;
  using K = SinK<R>;
  const int kl = A.KL, ml = A.ML;
  const R rog = Ph::ROWATER * Ph::G;
  const R const1 = A.BETAMAX / (Ph::XKAPPA * Ph::XKAPPA) / Ph::ROWATER;
  const R nu = Ph::RNUAIR;
  const R delabm1 = R(200) / (R(8.0) - R(0.3));
  const R shelter = mabs(A.TAUWSHELTER);
  T sig_n = wsigstar(P, USTAR, Z0);
  T uo = R(0), ao = R(0);
  for (int m = 0; m < ml; ++m) {
    T t = R(0);
    for (int k = 0; k < kl; ++k) t = t + F[k + kl * m];
    R sig = Ph::ZPI * A.FR[m];
    uo = uo + A.DFIM[m] * (sig * sig) * t;
    ao = ao + A.DFIM[m] * t;
  }
  const R tiny = sizeof(R) == 4 ? R(FLT_MIN) : R(DBL_MIN);
  T uorbt = R(2.0) * msqrt(tiny + uo);
  T aorb = R(2.0) * msqrt(tiny + ao);
  T re = (R(4.0) / nu) * uorbt * aorb;
  T z0noz = mmax(Ph::RNUAIRM / mmax(USTAR, R(0.0001)), R(0.04) * mmin(R(0.0005), Z0));
  T xi = (mlog10(mmax(aorb / z0noz, R(3.0))) - R(0.3)) * delabm1;
  int ind = (int)val(xi);
  ind = ind < 1 ? 1 : (ind > 199 ? 199 : ind);
  T deli1 = mmin(R(1.0), xi - R(ind));
  T fww = A.SWELLFT[ind - 1] * (R(1.0) - deli1) + A.SWELLFT[ind] * deli1;
  T temp2 = fww * uorbt;
  T smooth = R(0.5) * mtanh((re - K::SWELLF4) / K::SWELLF7);
  T pturb = R(0.5) + smooth, pvisc = R(0.5) - smooth;
  T usg[2] = {(USTAR * (R(1.0) + sig_n)) * (USTAR * (R(1.0) + sig_n)), (USTAR * (R(1.0) - sig_n)) * (USTAR * (R(1.0) - sig_n))};
  const R su = msin(P.UDIR), cu = mcos(P.UDIR);
  T taux[2] = {usg[0] * su, usg[1] * su}, tauy[2] = {usg[0] * cu, usg[1] * cu};
  T xst[2] = {R(0), R(0)}, yst[2] = {R(0), R(0)};
  const R rogoroair = rog / mmax(P.ROAIRN, R(1.0));
  T roairn_pvisc = P.ROAIRN * pvisc;
  for (int m = 0; m < ml; ++m) {
    tape[tape_sin(call, 0, ml) + m] = xst[0]; tape[tape_sin(call, 1, ml) + m] = xst[1];
    tape[tape_sin(call, 2, ml) + m] = yst[0]; tape[tape_sin(call, 3, ml) + m] = yst[1];
    const R sig = Ph::ZPI * A.FR[m], sig2 = sig * sig;
    R xk, cm;
    if (A.shallow) { xk = tfak(A, P, m); cm = xk * (R(1.0) / sig); }
    else { cm = sig / Ph::G; xk = sig2 / Ph::G; }
    T ustp[2], usdirp[2], ucn[2], ucnz[2];
    for (int g = 0; g < 2; ++g) {
      T tpx = taux[g] - shelter * xst[g], tpy = tauy[g] - shelter * yst[g];
      ustp[g] = mpow(tpx * tpx + tpy * tpy, R(0.25));
      usdirp[g] = matan2(tpx, tpy);
      ucn[g] = ustp[g] * cm;
      ucnz[g] = Ph::XKAPPA / (ucn[g] + A.ZALP);
    }
    const R constf = rogoroair * cm * A.DFIM[m];
    T zcn = mlog(xk * Z0);
    const R cnsn = (sig * const1) * P.ROAIRN;
    const R coef = -(K::SWELLF * R(16.) * sig2 / (Ph::G * Ph::ROWATER));
    const R coef5 = -(K::SWELLF5 * R(2.) * msqrt(R(2.) * nu * sig) / Ph::ROWATER);
    T dstab1 = coef5 * roairn_pvisc * xk;
    const R tmp1 = coef * P.ROAIRN;
    T px[2] = {R(0), R(0)}, py[2] = {R(0), R(0)}, st = R(0), sx = R(0), sy = R(0);
    for (int k = 0; k < kl; ++k) {
      const int b = k + kl * m;
      T f = F[b];
      T slp[2], flp[2];
      uint8_t ll = 0;
      for (int g = 0; g < 2; ++g) {
        T c = mcos(A.TH[k] - usdirp[g]);
        T ufac = R(0);
        if (c > R(0.01)) {
          T x = c * ucn[g], zlog = zcn + ucnz[g] / c;
          if (zlog < R(0.0)) { T z2x = zlog * zlog * x; ufac = mexp(zlog) * z2x * z2x; ll = 1; }
        }
        T dstab = dstab1 + pturb * (tmp1 * (temp2 + (K::FU + K::FUD * c) * ustp[g]));
        slp[g] = cnsn * ufac;
        flp[g] = slp[g] + dstab;
        slp[g] = slp[g] * f;
        px[g] = px[g] + slp[g] * (constf * A.SINTH[k]);
        py[g] = py[g] + slp[g] * (constf * A.COSTH[k]);
      }
      T spos = R(0.5) * (slp[0] + slp[1]);
      st = st + spos; sx = sx + spos * A.SINTH[k]; sy = sy + spos * A.COSTH[k];
      T fl = R(0.5) * (flp[0] + flp[1]);
      FL[b] = fl;
      SL[b] = fl * f;
      LL[b] = ll;
    }
    for (int g = 0; g < 2; ++g) { xst[g] = xst[g] + px[g]; yst[g] = yst[g] + py[g]; }
    tape[tape_sin(call, 4, ml) + m] = st; tape[tape_sin(call, 5, ml) + m] = sx; tape[tape_sin(call, 6, ml) + m] = sy;
  }
}

// TAU_PHI_HF (:3853-3966): high-frequency tail of the stress and energy flux.
template <typename R, typename T>
WAHD void tau_phi_hf(const ATabs<R>& A, int mij, T ustar, T z0, T& tauhf, T& phihf) {
  using Ph = Phys<R>;
  const R gm1 = R(1.0) / Ph::G;
  const R omegac = Ph::ZPI * A.FR[mij - 1];
  T tauw = ustar * ustar, ust = ustar;
  T xloggz0 = mlog(Ph::G * z0);
  T omegacc = mmax(omegac, A.X0TAUHF * Ph::G / ustar);
  T sqrtz0og = msqrt(z0 * gm1), sqrtgz0 = R(1.0) / sqrtz0og;
  T zinf = mlog(omegacc * sqrtz0og);
  T delz = mmax((R(0.0) - zinf) / R(18), R(0.0));
  tauhf = R(0); phihf = R(0);
  for (int j = 0; j < 19; ++j) {
    T y = mexp(zinf + R(j) * delz);
    T cm1 = y * sqrtgz0 * gm1;
    T zlog = mmin(xloggz0 + R(2.0) * mlog(cm1) + Ph::XKAPPA / (ust * cm1 + A.ZALP), R(0.0));
    T z2 = zlog * zlog;
    T fnc2 = mexp(zlog) * (z2 * z2) * tauw * A.WTAUHF[j] * delz;
    ust = msqrt(tauw);
    tauhf = tauhf + fnc2;
    phihf = phihf + fnc2 / y;
  }
  phihf = sqrtz0og * phihf;
}

template <typename R> WAHD R rhowgdfth(const ATabs<R>& A, int m, int mij) {
  const R rw = A.RHOWG[m];
  return (m == mij - 1 && mij != A.ML) ? R(0.5) * rw : rw;
}
template <typename R> WAHD R cmw(const ATabs<R>& A, const PointIn<R>& P, int m) {
  using Ph = Phys<R>;
  return A.shallow ? tfak(A, P, m) * (R(1.0) / (Ph::ZPI * A.FR[m])) : (Ph::ZPI * A.FR[m]) * (R(1.0) / Ph::G);
}

// STRESSO (:3164-3356) from SINPUT's per-frequency sums (tape) and the
// spectrum at the cut-off frequency.
template <typename R, typename T, typename FC>
WAHD T stresso(const ATabs<R>& A, const PointIn<R>& P, FC F, int mij, T USTAR, T Z0, Col<T> tape, int call) {
  using Ph = Phys<R>;
  const int kl = A.KL, ml = A.ML;
  T pphi = R(0), px = R(0), py = R(0);
  for (int m = 0; m < mij; ++m) {
    const R rw = rhowgdfth(A, m, mij), cmr = cmw(A, P, m) * rw;
    pphi = pphi + tape[tape_sin(call, 4, ml) + m] * rw;
    px = px + tape[tape_sin(call, 5, ml) + m] * cmr;
    py = py + tape[tape_sin(call, 6, ml) + m] * cmr;
  }
  const R gm1 = R(1.0) / Ph::G;
  const R cst = A.DELTH * ((Ph::ZPI * Ph::ZPI) * (Ph::ZPI * Ph::ZPI)) * gm1;
  T t1 = R(0), t2 = R(0);
  for (int k = 0; k < kl; ++k) {
    const R cw = mmax(mcos(A.TH[k] - P.UDIR), R(0.));
    T f = F[k + kl * (mij - 1)];
    t2 = t2 + f * (cw * cw);
    t1 = t1 + f * (cw * cw * cw);
  }
  T tau1, phi1;
  tau_phi_hf(A, mij, USTAR, Z0, tau1, phi1);
  T tauhf = cst * A.FR5[mij - 1] * gm1 * t1 * tau1;
  T xs = px / Ph::ROAIR + tauhf * msin(P.UDIR);
  T ys = py / Ph::ROAIR + tauhf * mcos(P.UDIR);
  T tw = msqrt(xs * xs + ys * ys);
  tw = mmin(tw, USTAR * USTAR - R(0.00001));
  return mmax(tw, R(0.));
}

// FRCUTINDEX (:3569-3647): the cut-off frequency index (a discrete decision).
template <typename R> WAHD int frcutindex(const ATabs<R>& A, R fm, R fmws, R ustar) {
  using Ph = Phys<R>;
  R fpmh = R(2.5) / A.FR[0];
  R fppm = R(3.0) * Ph::G / (R(28.0) * Ph::ZPI * A.FR[0]);
  R fpm4 = mmax(mmax(fmws, fm) * fpmh, fppm / mmax(ustar, R(1.0E-6)));
  int mij = (int)lround((double)(mlog10(fpm4) * A.INV_LOG_CO)) + 1;
  return mij < 1 ? 1 : (mij > A.ML ? A.ML : mij);
}

// IMPHFTAIL ratio of row m to row mij-1 (:3651-3731).
template <typename R> WAHD R tail_ratio_row(const ATabs<R>& A, const PointIn<R>& P, int m) {
  if (A.shallow) { R akm1 = R(1.) / tfak(A, P, m); return (akm1 * akm1 * akm1) / tcgond(A, P, m); }
  return A.FRM5[m];
}
template <typename R, typename T> WAHD void imphftail(const ATabs<R>& A, const PointIn<R>& P, Col<T> F, int mij) {
  const int kl = A.KL;
  const R base = tail_ratio_row(A, P, mij - 1);
  for (int m = mij; m < A.ML; ++m) {
    const R r = tail_ratio_row(A, P, m) / base;
    for (int k = 0; k < kl; ++k) F[k + kl * m] = r * F[k + kl * (mij - 1)];
  }
}

// SDISSIP_ARD (:1704-1962), SSDSC3 = SSDSC5 = 0.
template <typename R> WAHD R sds_facsat(const ATabs<R>& A, const PointIn<R>& P, int m) {
  using Ph = Phys<R>;
  const R sig = Ph::ZPI * A.FR[m];
  if (A.shallow) { R xk = tfak(A, P, m); return (xk * xk * xk) * (R(1.0) / Ph::ZPI) * tcgond(A, P, m); }
  R xk = sig * sig / Ph::G;
  return (xk * xk * xk) * (R(0.5) * (R(1.0) / Ph::ZPI)) * Ph::G / sig;
}
template <typename R, typename T>
WAHD void sdissip(const ATabs<R>& A, const PointIn<R>& P, Col<T> F, Col<T> SL, Col<T> FL) {
  using Ph = Phys<R>;
  const int kl = A.KL, nw = 2 * A.NSDSNTH + 1;
  const R tmp03 = R(1.0) / R(9.0E-4), c6 = R(0.3), c6m1 = R(1.) - c6;
  T bth[MAX_KL];
  for (int m = 0; m < A.ML; ++m) {
    const R facsat = sds_facsat(A, P, m), ssdsc2_sig = R(-2.2E-5) * (Ph::ZPI * A.FR[m]);
    T bmax = R(0);
    for (int k = 0; k < kl; ++k) {
      T acc = R(0);
      for (int j = 0; j < nw; ++j) acc = acc + A.SATW[k + kl * j] * F[(A.INDSAT[k + kl * j] - 1) + kl * m];
      bth[k] = acc * facsat;
      bmax = mmax(bmax, bth[k]);
    }
    T d0 = mmax(R(0.), bmax * tmp03 - R(1.0));
    T temp1 = c6 * (d0 * d0);
    for (int k = 0; k < kl; ++k) {
      const int b = k + kl * m;
      T dd = mmax(R(0.), bth[k] * tmp03 - R(1.0));
      T d = ssdsc2_sig * (temp1 + c6m1 * (dd * dd));
      SL[b] = SL[b] + d * F[b];
      FL[b] = FL[b] + d;
    }
  }
}

// SNONLIN (DIA, :2742-3047) in the reference's loop order.
template <typename R, typename T>
WAHD T snl_enhfr(const ATabs<R>& A, const PointIn<R>& P, T AKMEAN) {
  T e = mmax(R(0.75) * P.DEPTH * AKMEAN, R(.5));
  return R(1.) + (R(5.5) / e) * (R(1.) - R(.833) * e) * mexp(R(-1.25) * e);
}


// One DIA interaction (MC, KH, K): the 9 gathered bins and the 9 target bins
// with their write masks (the MC regimes of :2890, :2942, :2999).
template <typename R> struct DiaInt {
  int mc;
  int iC, iP, iP_11, iP1, iP1_11, iM, iM_21, iM1, iM1_21;   // gathered: centre, K1W/K11W at IP/IP1, K2W/K21W at IM/IM1
  int tC, tMM, tMM1, tMP, tMP1, tMM_21, tMM1_21, tMP_11, tMP1_11;  // targets
  bool wMC, wMM, wMM1, wMP, wMP1;
  R g[8], ftail, af11;
  const R* rc;
};

template <typename R, class Fn> WAHD void dia_for_each(const ATabs<R>& A, Fn&& fn) {
  const int kl = A.KL, ml = A.ML;
  const int mfr1 = -A.MFRSTLW + 1, mfrl = ml - A.KFRH + mfr1;
  DiaInt<R> d;
  for (int mc = 1; mc <= A.MLSTHG; ++mc) {
    const int im = mc - A.MFRSTLW;
    const int MP = A.IKP[im], MP1 = A.IKP1[im], MM = A.IKM[im], MM1 = A.IKM1[im];
    const int* ic5 = A.INL + 5 * (mc - 1);
    const R* rc = A.RNL + RNL_STRIDE * (mc - 1);
    const int regime = (mc > mfr1 && mc < mfrl) ? 0 : (mc >= mfrl ? 1 : 2);
    d.mc = mc; d.rc = rc; d.af11 = A.AF11[im];
    d.ftail = (regime == 0) ? R(1) : rc[0];
    d.wMM = regime != 2;
    d.wMM1 = regime == 0 || (regime == 1 && MM1 <= ml) || (regime == 2 && MM1 >= 1);
    d.wMC = regime != 1 || (MM1 <= ml && mc <= ml);
    d.wMP = regime != 1 || (MM1 <= ml && mc <= ml && MP <= ml);
    d.wMP1 = regime != 1 || (MM1 <= ml && mc <= ml && MP <= ml && MP1 <= ml);
    const int g_idx[8] = {1, 2, 3, 4, 13, 14, 15, 16};
    for (int q = 0; q < 8; ++q) d.g[q] = rc[rnl_slot(g_idx[q])];
    for (int kh = 0; kh < 2; ++kh)
      for (int k = 0; k < kl; ++k) {
        const int a1 = A.K1W[k + kl * kh] - 1, a2 = A.K2W[k + kl * kh] - 1, a11 = A.K11W[k + kl * kh] - 1,
                  a21 = A.K21W[k + kl * kh] - 1;
        d.iC = k + kl * (ic5[0] - 1);
        d.iP = a1 + kl * (ic5[1] - 1); d.iP_11 = a11 + kl * (ic5[1] - 1);
        d.iP1 = a1 + kl * (ic5[2] - 1); d.iP1_11 = a11 + kl * (ic5[2] - 1);
        d.iM = a2 + kl * (ic5[3] - 1); d.iM_21 = a21 + kl * (ic5[3] - 1);
        d.iM1 = a2 + kl * (ic5[4] - 1); d.iM1_21 = a21 + kl * (ic5[4] - 1);
        d.tC = k + kl * (mc - 1);
        d.tMM = a2 + kl * (MM - 1); d.tMM1 = a2 + kl * (MM1 - 1); d.tMP = a1 + kl * (MP - 1); d.tMP1 = a1 + kl * (MP1 - 1);
        d.tMM_21 = a21 + kl * (MM - 1); d.tMM1_21 = a21 + kl * (MM1 - 1);
        d.tMP_11 = a11 + kl * (MP - 1); d.tMP1_11 = a11 + kl * (MP1 - 1);
        fn(d);
      }
  }
}

template <typename R, typename T> WAHD T dia_ftemp(const ATabs<R>& A, const PointIn<R>& P, const DiaInt<R>& d, T enhfr) {
  T ftemp = T(d.af11);
  if (A.shallow) ftemp = ftemp * (A.isnonlin == 0 ? enhfr : T(P.ENH[d.mc - 1]));
  return ftemp;
}

template <typename R, typename T>
WAHD void snonlin(const ATabs<R>& A, const PointIn<R>& P, Col<T> F, T AKMEAN, Col<T> SL, Col<T> FL) {
  const T enhfr = (A.shallow && A.isnonlin == 0) ? snl_enhfr(A, P, AKMEAN) : T(R(1));
  dia_for_each(A, [&](const DiaInt<R>& d) {
    const R* rc = d.rc;
    T sap = d.g[0] * F[d.iP] + d.g[1] * F[d.iP_11] + d.g[2] * F[d.iP1] + d.g[3] * F[d.iP1_11];
    T sam = d.g[4] * F[d.iM] + d.g[5] * F[d.iM_21] + d.g[6] * F[d.iM1] + d.g[7] * F[d.iM1_21];
    T fij = F[d.iC] * d.ftail;
    T fad1 = fij * (sap + sam);
    T fad2 = fad1 - R(2.) * sap * sam;
    fad1 = fad1 + fad2;
    const T ftemp = dia_ftemp(A, P, d, enhfr);
    T fcen = ftemp * fij;
    T ad = fad2 * fcen, delad = fad1 * ftemp;
    T delap = (fij - R(2.) * sam) * A.DAL1 * fcen, delam = (fij - R(2.) * sap) * A.DAL2 * fcen;
    if (d.wMC) { SL[d.tC] = SL[d.tC] - R(2.) * ad; FL[d.tC] = FL[d.tC] - R(2.) * delad; }
    if (d.wMM) {
      SL[d.tMM] = SL[d.tMM] + ad * rc[rnl_slot(20)]; FL[d.tMM] = FL[d.tMM] + delam * rc[rnl_slot(23)];
      SL[d.tMM_21] = SL[d.tMM_21] + ad * rc[rnl_slot(19)]; FL[d.tMM_21] = FL[d.tMM_21] + delam * rc[rnl_slot(24)];
    }
    if (d.wMM1) {
      SL[d.tMM1] = SL[d.tMM1] + ad * rc[rnl_slot(17)]; FL[d.tMM1] = FL[d.tMM1] + delam * rc[rnl_slot(21)];
      SL[d.tMM1_21] = SL[d.tMM1_21] + ad * rc[rnl_slot(18)]; FL[d.tMM1_21] = FL[d.tMM1_21] + delam * rc[rnl_slot(22)];
    }
    if (d.wMP) {
      SL[d.tMP] = SL[d.tMP] + ad * rc[rnl_slot(8)]; FL[d.tMP] = FL[d.tMP] + delap * rc[rnl_slot(11)];
      SL[d.tMP_11] = SL[d.tMP_11] + ad * rc[rnl_slot(7)]; FL[d.tMP_11] = FL[d.tMP_11] + delap * rc[rnl_slot(12)];
    }
    if (d.wMP1) {
      SL[d.tMP1] = SL[d.tMP1] + ad * rc[rnl_slot(5)]; FL[d.tMP1] = FL[d.tMP1] + delap * rc[rnl_slot(9)];
      SL[d.tMP1_11] = SL[d.tMP1_11] + ad * rc[rnl_slot(6)]; FL[d.tMP1_11] = FL[d.tMP1_11] + delap * rc[rnl_slot(10)];
    }
  });
}

// SBOTTOM factor per frequency (:1527-1589), depth only.
template <typename R> WAHD R sbottom(const ATabs<R>& A, const PointIn<R>& P, int m) {
  using Ph = Phys<R>;
  const R cst = R(-2.0) * R(0.038) / Ph::G;
  const R wav = tfak(A, P, m);
  return cst * wav / msinh(mmin(R(2.) * P.DEPTH * wav, R(50.)));
}

// The implicit integration with the growth limiter and the minimum-energy
// floor (:640-670), in place on Fw (F1 in, F2 out).
template <typename R, typename T>
WAHD void update(const ATabs<R>& A, const PointIn<R>& P, Col<T> Fw, Col<T> SL, Col<T> FL, T USTAR, T fmx, int ju) {
  const int kl = A.KL;
  for (int m = 0; m < A.ML; ++m) {
    const R sbo = A.shallow ? sbottom(A, P, m) : R(0);
    T lim = USTAR * A.DELFL[m] * fmx;
    const R fmin = A.FLMINFR[(ju - 1) + 300 * m];
    for (int k = 0; k < kl; ++k) {
      const int b = k + kl * m;
      const R c = mmax(R(0.), mcos(A.TH[k] - P.UDIR));
      T f0 = Fw[b], sl = SL[b], fl = FL[b];
      if (A.shallow) { sl = sl + sbo * f0; fl = fl + sbo; }
      T t1 = A.DELT * sl / mmax(R(1.), R(1.) - A.DELT * fl);
      T t3 = mmin(mabs(t1), lim);
      T f = f0 + ((t1 >= R(0)) ? t3 : -t3);
      Fw[b] = mmax(f, fmin * (c * c));
    }
  }
}

// The whole IMPLSCH step of one point, ST4 (:374-700).  F0 is the input
// spectrum; Fw receives the output (and holds F after each stage on the way).
template <typename R, typename T>
WAHD void forward(const ATabs<R>& A, const PointIn<R>& P, Col<const T> F0, T TAUW0, T U10, Col<T> Fw, Col<T> SL,
                  Col<T> FL, Col<uint8_t> LL1, Col<uint8_t> LL, Col<T> tape, int* itape, T& TAUW, T& USTAR, T& Z0) {
  const int n = A.KL * A.ML;
  const Col<const uint8_t> nomask{nullptr, 0}, llc1{LL1.p, LL1.ld}, llc{LL.p, LL.ld};
  for (int b = 0; b < n; ++b) Fw[b] = F0[b];
  int ju = (int)lround((double)(val(U10) / A.DELU));
  ju = ju < 1 ? 1 : (ju > 300 ? 300 : ju);
  T emean, fmean, akmean = R(0), emeanws, fmeanws;
  const bool need_ak = A.shallow && A.isnonlin == 0;
  integrals(A, P, Fw, nomask, emean, fmean, need_ak ? &akmean : nullptr);
  T us1, z01;
  airsea(A, U10, TAUW0, us1, z01);
  sinput(A, P, Fw, us1, z01, SL, FL, LL1, tape, 0);
  integrals(A, P, Fw, llc1, emeanws, fmeanws, (T*)nullptr);
  const int mij = frcutindex(A, val(fmean), val(fmeanws), val(us1));
  T tauw1 = stresso(A, P, Fw, mij, us1, z01, tape, 0);
  T us2, z02;
  airsea(A, U10, tauw1, us2, z02);
  imphftail(A, P, Fw, mij);
  sinput(A, P, Fw, us2, z02, SL, FL, LL, tape, 1);
  T tauw2 = stresso(A, P, Fw, mij, us2, z02, tape, 1);
  sdissip(A, P, Fw, SL, FL);
  snonlin(A, P, Fw, akmean, SL, FL);
  update(A, P, Fw, SL, FL, us2, mmax(fmeanws, fmean), ju);
  T e2, fm2, ews2, fmws2;
  integrals(A, P, Fw, nomask, e2, fm2, (T*)nullptr);
  integrals(A, P, Fw, llc, ews2, fmws2, (T*)nullptr);
  const int mij2 = frcutindex(A, val(fm2), val(fmws2), val(us2));
  imphftail(A, P, Fw, mij2);
  const int ml = A.ML;
  tape[tape_scalar(TS_USTAR1, ml)] = us1; tape[tape_scalar(TS_Z01, ml)] = z01; tape[tape_scalar(TS_TAUW1, ml)] = tauw1;
  tape[tape_scalar(TS_USTAR2, ml)] = us2; tape[tape_scalar(TS_Z02, ml)] = z02; tape[tape_scalar(TS_TAUW2, ml)] = tauw2;
  tape[tape_scalar(TS_EMEAN, ml)] = emean; tape[tape_scalar(TS_FMEAN, ml)] = fmean;
  tape[tape_scalar(TS_AKMEAN, ml)] = akmean; tape[tape_scalar(TS_EMEANWS, ml)] = emeanws;
  tape[tape_scalar(TS_FMEANWS, ml)] = fmeanws;
  itape[TI_MIJ] = mij; itape[TI_MIJ2] = mij2; itape[TI_JU] = ju;
  TAUW = tauw2; USTAR = us2; Z0 = z02;
}


// ---- derivatives of the scalar routines ------------------------------------------

// Jacobian of a scalar routine with two inputs (d out_i / d in_j).
template <typename R> struct Jac2 { R d00, d01, d10, d11; };

}  // namespace adj
}  // namespace wamgpu
