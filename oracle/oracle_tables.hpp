// ORACLE — test infrastructure only. Never linked into, imported by, or called
// from the wam_b200 product library. It is the CPU checker that the GPU kernels
// are compared against in tests/ and the timed CPU baseline leg of bench.py.
//
// This file restates, statement by statement, the static-table builders of
// myWAveModel/WAM Cycle 7 (GPL-3.0; file:line citations are relative to the
// reference project root).  The restatement keeps the reference's loop order,
// operand association and single-precision literals, so that with R=float it
// reproduces the Fortran REAL arithmetic (no -ffast-math, no FMA contraction).
// With R=double it is the FP64 run of the same algorithm.
//
// Parity pins: the DIA index/weight tables, the frequency grid and the tail
// table are checked against the run protocol dayfiles/wam_prot_coarse_ST6:
// 322-346 and 876-936 (tests/test_oracle_golden.py).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include <stdexcept>
#include <limits>

namespace wamo {

// ---- Fortran intrinsic helpers ------------------------------------------
template <typename R> inline R ipow(R x, int n) {
  // Fortran REAL**INTEGER: binary powering, negative exponents by reciprocal.
  if (n < 0) return R(1) / ipow(x, -n);
  R result = R(1); bool first = true; R base = x;
  while (n > 0) {
    if (n & 1) { result = first ? base : result * base; first = false; }
    n >>= 1;
    if (n) base = base * base;
  }
  return result;
}
// Correctly rounded REAL intrinsics for the values that decide an integer:
// the cut-off index MIJ (LOG10 in FRCUTINDEX, LOG in FRCUTINDEX_ST6), the
// LFACTOR iteration (EXP, and COS/SIN of the wind direction) and the
// wavenumbers and group velocities of WAVNU2 that enter it (TANH, COSH, SINH).  The Fortran
// standard leaves the accuracy of LOG10, EXP, ... processor dependent; glibc's
// single-precision log10f, for one, is off by one ulp for about 7% of its
// arguments.  Evaluating these few per-point values in double and rounding
// once gives the correctly rounded REAL result, which the GPU kernels compute
// the same way, so equal inputs give equal decisions on both sides.
template <typename R> inline R crlog10(R x) { return R(std::log10((double)x)); }
template <typename R> inline R crlog(R x) { return R(std::log((double)x)); }
template <typename R> inline R crexp(R x) { return R(std::exp((double)x)); }
template <typename R> inline R crcos(R x) { return R(std::cos((double)x)); }
template <typename R> inline R crsin(R x) { return R(std::sin((double)x)); }
template <typename R> inline R crtanh(R x) { return R(std::tanh((double)x)); }
template <typename R> inline R crcosh(R x) { return R(std::cosh((double)x)); }
template <typename R> inline R crsinh(R x) { return R(std::sinh((double)x)); }
inline int nint_f(double x) { return (int)std::lround(x); }           // NINT
inline int int_f(double x) { return (int)std::trunc(x); }            // INT
template <typename R> inline R fsign(R a, R b) { return b >= R(0) ? std::fabs(a) : -std::fabs(a); }

// wam_general_module.f90:41-124 (REAL PARAMETERs, single precision folding)
template <typename R> struct K {
  static constexpr R G = R(9.806);
  static constexpr R PI = R(3.1415927);
  static constexpr R ZPI = R(2.) * PI;
  static constexpr R DEG = R(180.) / PI;
  static constexpr R RAD = PI / R(180.);
  static constexpr R CIRC = R(40000000.);
  static constexpr R REARTH = CIRC / ZPI;
  static constexpr R ROAIR = R(1.225);
  static constexpr R RNUAIR = R(1.5E-5);
  static constexpr R RNUAIRM = R(0.11) * RNUAIR;
  static constexpr R ROWATER = R(1000.);
  static constexpr R XEPS = ROAIR / ROWATER;
  static constexpr R XKAPPA = R(0.40);
  static constexpr R XNLEV = R(10.0);
  static constexpr R DKMAX = R(40.);
  static constexpr R SDSBR = R(9.0E-4);
  static constexpr int ISDSDTH = 80;
  static constexpr int ISB = 2;
  static constexpr int IPSAT = 2;
  static constexpr R SSDSC2 = R(-2.2E-5);
  static constexpr R SSDSC4 = R(1.0);
  static constexpr R SSDSC6 = R(0.3);
  static constexpr R MICHE = R(1.0);
  // wam_tables_module.f90:57-66
  static constexpr R FETCH_MAX = R(25000.);
  static constexpr R FLMIN = R(0.000001);
  static constexpr int JUMAX = 300;
  static constexpr R UMAX = R(75.);
  static constexpr R EPS1 = R(0.00001);
  // wam_interface_module.f90:44
  static constexpr R EMIN = R(1.0E-12);
  // wam_fre_dir_module.f90:42,45
  static constexpr R CO = R(1.1);
  static constexpr int EX_TAIL = -5;
};

// Model configuration mirrored from the reference's module flags
// (wam_timopt_module.f90, wam_general_module.f90:63-74, initmdl.f90:153-160).
struct OracleConfig {
  int kl, ml;
  double fr1; int iref;
  int iphys;              // 1 = ST4 (ARD), 2 = ST6
  int shallow_run, spherical_run, refraction_d_run, refraction_c_run, reduced_grid;
  int isnonlin, lcflx;
  int idelt, idelpro;
  double betamax, zalp, alpha, tauwshelter, cdfac;
  int ndepth; double deptha, depthd;
  double delphi;          // latitude increment [m] (MIN_ENERGY fetch, propagation)
};

// ---- frequency/direction grid: wam_fre_dir_module.f90:297-459 -------------
template <typename R> struct FreDir {
  int KL, ML;
  std::vector<R> FR, DF, DF_FR, DF_FR2, DFIM, DFIMOFR, DFIM_FR, DFIM_FR2, FR5, FRM5,
      RHOWG_DFIM, GOM, C, TH, COSTH, SINTH;
  R DELTH, DELTR, INV_LOG_CO, MO_TAIL, MM1_TAIL, MP1_TAIL, MP2_TAIL, FMIN;
  std::vector<int> MPM, KPM, JXO, JYO;  // MPM[m*3+(d+1)], KPM[k*3+(d+1)], JXO[k*2+i]

  void build(int kl, int ml, R fr1, int iref) {
    using C_ = K<R>;
    KL = kl; ML = ml;
    FR.assign(ML, 0);
    FR[0] = ipow(C_::CO, -iref + 1) * fr1;                     // fre_dir:212
    INV_LOG_CO = R(1.) / std::log10(C_::CO);                   // :312
    for (int m = 1; m < ML; ++m) FR[m] = C_::CO * FR[m - 1];   // :314-316
    FR5.resize(ML); FRM5.resize(ML);
    for (int m = 0; m < ML; ++m) { FR5[m] = ipow(FR[m], 5); FRM5[m] = R(1) / FR5[m]; }
    GOM.resize(ML); C.resize(ML);
    for (int m = 0; m < ML; ++m) {
      GOM[m] = C_::G / ((R(2.) * C_::ZPI) * FR[m]);            // :330
      C[m] = C_::G / (C_::ZPI * FR[m]);                         // :338
    }
    DELTH = C_::ZPI / R(KL);                                    // :345
    DELTR = DELTH * C_::REARTH;
    TH.resize(KL); COSTH.resize(KL); SINTH.resize(KL);
    for (int k = 0; k < KL; ++k) TH[k] = R(k) * DELTH + R(0.5) * DELTH;  // :355
    for (int k = 0; k < KL; ++k) { COSTH[k] = std::cos(TH[k]); SINTH[k] = std::sin(TH[k]); }
    R CO1 = R(0.5) * (C_::CO - R(1.));                          // :377
    DF.resize(ML);
    DF[0] = CO1 * FR[0];
    for (int m = 1; m < ML - 1; ++m) DF[m] = CO1 * (FR[m] + FR[m - 1]);
    DF[ML - 1] = CO1 * FR[ML - 2];
    DF_FR.resize(ML); DF_FR2.resize(ML);
    for (int m = 0; m < ML; ++m) { DF_FR[m] = DF[m] * FR[m]; DF_FR2[m] = DF_FR[m] * FR[m]; }
    DFIM.resize(ML); DFIMOFR.resize(ML); DFIM_FR.resize(ML); DFIM_FR2.resize(ML); RHOWG_DFIM.resize(ML);
    const R ROG = C_::ROWATER * C_::G;
    for (int m = 0; m < ML; ++m) {
      DFIM[m] = DF[m] * DELTH;                                  // :391
      DFIMOFR[m] = DFIM[m] / FR[m];
      DFIM_FR[m] = DF_FR[m] * DELTH;
      DFIM_FR2[m] = DF_FR2[m] * DELTH;
      RHOWG_DFIM[m] = ((ROG * DELTH) * std::log(C_::CO)) * FR[m];  // :395
    }
    RHOWG_DFIM[0] = R(0.5) * RHOWG_DFIM[0];
    RHOWG_DFIM[ML - 1] = R(0.5) * RHOWG_DFIM[ML - 1];
    MO_TAIL = -(DELTH / R(C_::EX_TAIL + 1) * FR[ML - 1]);          // :406
    MM1_TAIL = -(DELTH / R(C_::EX_TAIL));
    MP1_TAIL = -(DELTH / R(C_::EX_TAIL + 2) * ipow(FR[ML - 1], 2));
    MP2_TAIL = -(DELTH / R(C_::EX_TAIL + 3) * ipow(FR[ML - 1], 3));
    FMIN = ipow(R(0.07), 2) / ((R(16.) * (FR[ML - 1] - FR[0])) * C_::ZPI);  // :416
    MPM.assign(ML * 3, 0);
    for (int m = 1; m <= ML; ++m) {                              // :424-428 (1-based values)
      MPM[(m - 1) * 3 + 0] = std::max(1, m - 1);
      MPM[(m - 1) * 3 + 1] = m;
      MPM[(m - 1) * 3 + 2] = std::min(ML, m + 1);
    }
    KPM.assign(KL * 3, 0); JXO.assign(KL * 2, 0); JYO.assign(KL * 2, 0);
    for (int k = 1; k <= KL; ++k) {                              // :434-457
      int km = k - 1; if (km < 1) km = KL;
      int kp = k + 1; if (kp > KL) kp = 1;
      KPM[(k - 1) * 3 + 0] = km; KPM[(k - 1) * 3 + 1] = k; KPM[(k - 1) * 3 + 2] = kp;
      if (COSTH[k - 1] >= R(0.)) { JYO[(k - 1) * 2] = 1; JYO[(k - 1) * 2 + 1] = 2; }
      else { JYO[(k - 1) * 2] = 2; JYO[(k - 1) * 2 + 1] = 1; }
      if (SINTH[k - 1] >= R(0.)) { JXO[(k - 1) * 2] = 1; JXO[(k - 1) * 2 + 1] = 2; }
      else { JXO[(k - 1) * 2] = 2; JXO[(k - 1) * 2 + 1] = 1; }
    }
  }
};

// ---- AKI: wam_general_module.f90:301-364 ----------------------------------
template <typename R> R AKI(R OM, R BETA) {
  using C_ = K<R>;
  const R EBS = R(0.0001);
  R aki = std::max(ipow(OM, 2) / (R(4.) * C_::G), OM / (R(2.) * std::sqrt(C_::G * BETA)));
  R AKP = R(10000.);
  while (std::fabs(AKP - aki) > EBS * aki) {
    R BO = BETA * aki;
    if (BO > C_::DKMAX) { aki = ipow(OM, 2) / C_::G; break; }
    AKP = aki;
    R TH = (C_::G * aki) * std::tanh(BO);
    R STH = std::sqrt(TH);
    aki = aki + (OM - STH) * STH * R(2.) / (TH / aki + C_::G * BO / ipow(std::cosh(BO), 2));
  }
  return aki;
}

// ---- TRANSF: wam_interface_module.f90:2614-2680 ---------------------------
template <typename R> R TRANSF(R XK, R D) {
  using C_ = K<R>;
  const R EPS = R(0.0001);
  if (D < R(999.) && D > R(0.)) {
    R X = XK * D;
    if (X > C_::DKMAX) return R(1.);
    R T_0 = std::tanh(X);
    R OM = std::sqrt((C_::G * XK) * T_0);
    R C_0 = OM / XK;
    R V_G;
    if (X < EPS) { V_G = C_0; }
    else { V_G = (R(0.5) * C_0) * (R(1.) + R(2.) * X / std::sinh(R(2.) * X)); }
    R DV_G = ipow(T_0 - X * (R(1.) - ipow(T_0, 2)), 2) +
             ((R(4.) * ipow(X, 2)) * ipow(T_0, 2)) * (R(1.) - ipow(T_0, 2));
    R XNL_1 = ((R(9.) * ipow(T_0, 4) - R(10.) * ipow(T_0, 2)) + R(9.)) / (R(8.) * ipow(T_0, 3));
    R XNL_2 = (ipow(R(2.) * V_G - R(0.5) * C_0, 2) / (C_::G * D - ipow(V_G, 2)) + R(1.)) / X;
    R XNL = XNL_1 - XNL_2;
    return ipow(XNL, 2) / (DV_G * ipow(T_0, 8));
  }
  return R(1.);
}

// ---- shallow water tables: wam_tables_module.f90:388-464 ------------------
template <typename R> struct ShallowTables {
  int NDEPTH; R DEPTHA, DEPTHD;
  std::vector<R> TFAK, TCGOND, TSIHKD, TFAC_ST, T_TAIL;  // [(jd-1) + NDEPTH*(m-1)]
  void build(const FreDir<R>& fd, int ndepth, R deptha, R depthd) {
    using C_ = K<R>;
    NDEPTH = ndepth; DEPTHA = deptha; DEPTHD = depthd;
    int ML = fd.ML;
    TFAK.assign(NDEPTH * ML, 0); TCGOND = TFAK; TSIHKD = TFAK; TFAC_ST = TFAK; T_TAIL = TFAK;
    const R GH = C_::G / (R(4.) * C_::PI);
    for (int m = 0; m < ML; ++m) {
      R OM = C_::ZPI * fd.FR[m];
      for (int jd = 1; jd <= NDEPTH; ++jd) {
        R AD = DEPTHA * ipow(DEPTHD, jd - 1);
        R AK = AKI(OM, AD);
        size_t i = (jd - 1) + (size_t)NDEPTH * m;
        TFAK[i] = AK;
        R AKD = AK * AD;
        if (AKD <= R(10.0)) {
          TCGOND[i] = R(0.5) * std::sqrt(C_::G * std::tanh(AKD) / AK) * (R(1.0) + R(2.0) * AKD / std::sinh(R(2.) * AKD));
          TSIHKD[i] = OM / std::sinh(R(2.) * AKD);
          TFAC_ST[i] = R(2.) * C_::G * ipow(AK, 2) / (OM * std::tanh(R(2.) * AKD));
          T_TAIL[i] = R(1.) / (ipow(TFAK[i], 3) * TCGOND[i]);
        } else {
          TCGOND[i] = GH / fd.FR[m];
          TSIHKD[i] = R(0.);
          TFAC_ST[i] = R(2.) / C_::G * ipow(OM, 3);
          T_TAIL[i] = R(1.) / (ipow(TFAK[i], 3) * TCGOND[i]);
        }
      }
    }
  }
  R tfak(int jd, int m) const { return TFAK[(jd - 1) + (size_t)NDEPTH * m]; }      // jd 1-based, m 0-based
  R tcgond(int jd, int m) const { return TCGOND[(jd - 1) + (size_t)NDEPTH * m]; }
  R tsihkd(int jd, int m) const { return TSIHKD[(jd - 1) + (size_t)NDEPTH * m]; }
};

// ---- MIN_ENERGY + FETCH_LAW + JONSWAP: wam_tables_module.f90:315-384,
//      wam_jonswap_module.f90:63-211 ------------------------------------------
template <typename R> void fetch_law(R FETCH, R FPMAX, const std::vector<R>& U10, std::vector<R>& ALPHJ, std::vector<R>& FP) {
  using C_ = K<R>;
  const R A = R(2.84), D = -(R(3.) / R(10.)), B = R(0.033), E = R(2.) / R(3.);
  size_t n = U10.size(); ALPHJ.resize(n); FP.resize(n);
  for (size_t i = 0; i < n; ++i) {
    if (U10[i] > R(0.1E-08)) {
      R UG = C_::G / U10[i];
      R fp = std::max(R(0.13), A * std::pow((C_::G * FETCH) / ipow(U10[i], 2), D));
      fp = std::min(fp, FPMAX / UG);
      ALPHJ[i] = std::max(R(0.0081), B * std::pow(fp, E));
      FP[i] = fp * UG;
    } else { ALPHJ[i] = R(0.0081); FP[i] = FPMAX; }
  }
}
// ET[i + nfp*m]
template <typename R> void jonswap(const std::vector<R>& FR, const std::vector<R>& ALPHAJ, R GAMMA, R SA, R SB,
                                   const std::vector<R>& FP, std::vector<R>& ET) {
  using C_ = K<R>;
  size_t nfp = FP.size(), ML = FR.size();
  ET.assign(nfp * ML, 0);
  const R G2ZPI4 = ipow(C_::G, 2) / ipow(C_::ZPI, 4);
  R LOG_GAMMA = std::log(GAMMA);
  R SAA = R(0.5) / (SA * SA), SBB = R(0.5) / (SB * SB);
  for (size_t m = 0; m < ML; ++m) {
    R FRH = FR[m];
    R g2 = G2ZPI4 * ipow(FR[m], -5);
    for (size_t i = 0; i < nfp; ++i) {
      R ARG = R(1.25) * ipow(FP[i] / FRH, 4);
      R et;
      if (ARG < R(50.)) et = ALPHAJ[i] * g2 * std::exp(-ARG);
      else { ET[i + nfp * m] = R(0.); continue; }
      if (FRH > FP[i]) ARG = SBB * ipow(FRH / FP[i] - R(1.), 2);
      else ARG = SAA * ipow(FRH / FP[i] - R(1.), 2);
      if (ARG < R(99.)) et = et * std::exp(LOG_GAMMA * std::exp(-ARG));
      ET[i + nfp * m] = et;
    }
  }
}
template <typename R> struct MinEnergy {
  R DELU;
  std::vector<R> FLMINFR;  // [(ju-1) + JUMAX*m]
  void build(const FreDir<R>& fd, R DELPHI) {
    using C_ = K<R>;
    const int JUMAX = C_::JUMAX;
    std::vector<R> U10(JUMAX), FPK, ALPHJO;
    DELU = C_::UMAX / R(JUMAX);
    for (int j = 1; j <= JUMAX; ++j) U10[j - 1] = R(j) * DELU;
    R FETCH = std::min(R(0.5) * DELPHI, C_::FETCH_MAX);
    fetch_law(FETCH, fd.FR[fd.ML - 1], U10, ALPHJO, FPK);
    for (auto& a : ALPHJO) a = R(0.01) * a;
    jonswap(fd.FR, ALPHJO, R(3.000000), R(7.000000E-02), R(9.000000E-02), FPK, FLMINFR);
    for (auto& v : FLMINFR) v = std::max(v, C_::FLMIN);
  }
};

// ---- DIA tables: NLWEIGT (wam_source_module.f90:1056-1287), JAFU
//      (src/chief/jafu.f90:3-39), INIT_SNONLIN (:1291-1523) ----------------
inline int JAFU(double CL, int J, int IAN) {
  int j = J + int_f(CL);
  if (j <= 0) j += IAN;
  if (j > IAN) j -= IAN;
  return j;
}
template <typename R> struct DiaTables {
  int MFRSTLW, MLSTHG, KFRH, ISP, ISM;
  R ACL1, ACL2, CL11, CL21, DAL1, DAL2;
  // arrays indexed by M in [MFRSTLW, MLSTHG]: stored at [M - MFRSTLW]
  std::vector<int> IKP, IKP1, IKM, IKM1;
  std::vector<R> AF11, FKLAP, FKLAP1, FKLAM, FKLAM1;
  std::vector<int> K1W, K2W, K11W, K21W;  // [(k-1) + KL*(kh-1)]
  std::vector<R> FRH;                      // [0..KFRH-1]
  std::vector<R> FTRF;                     // index MC in [MFRSTLW,1]: [MC - MFRSTLW]
  std::vector<int> INLCOEF;                // [(i-1) + 5*(mc-1)], mc 1..MLSTHG
  std::vector<R> RNLCOEF;                  // [(i-1) + 25*(mc-1)]

  int ikp(int M) const { return IKP[M - MFRSTLW]; }
  int ikp1(int M) const { return IKP1[M - MFRSTLW]; }
  int ikm(int M) const { return IKM[M - MFRSTLW]; }
  int ikm1(int M) const { return IKM1[M - MFRSTLW]; }

  void build(const FreDir<R>& fd) {
    using C_ = K<R>;
    const int KL = fd.KL, ML = fd.ML;
    const R ALAMD = R(0.25), CON = R(3000.);
    R F1P1 = std::log10(C_::CO);
    ISP = int_f(std::log10(R(1.) + ALAMD) / F1P1 + R(.000001));
    ISM = (int)std::floor(std::log10(R(1.) - ALAMD) / F1P1 + R(.0000001));
    MFRSTLW = 1 + ISM;
    MLSTHG = ML - ISM;
    KFRH = -ISM + ISP + 2;
    std::vector<int> JA1(KL * 2), JA2(KL * 2);
    std::vector<R> FRLON(ML + KFRH - MFRSTLW + 1);
    auto frlon = [&](int M) -> R& { return FRLON[M - MFRSTLW]; };
    int n = MLSTHG - MFRSTLW + 1;
    IKP.assign(n, 0); IKP1 = IKP; IKM = IKP; IKM1 = IKP;
    AF11.assign(n, 0); FKLAP = AF11; FKLAP1 = AF11; FKLAM = AF11; FKLAM1 = AF11;
    K1W.assign(KL * 2, 0); K2W = K1W; K11W = K1W; K21W = K1W;
    FRH.assign(KFRH, 0);
    // :1153-1161
    R XF = ipow((R(1.) + ALAMD) / (R(1.) - ALAMD), 4);
    R COSTH3 = (R(1.) + R(2.) * ALAMD + R(2.) * ipow(ALAMD, 3)) / ipow(R(1.) + ALAMD, 2);
    R DELPHI1 = -(R(180.) / C_::PI * std::acos(COSTH3));
    R COSTH4 = std::sqrt(R(1.) - XF + XF * ipow(COSTH3, 2));
    R DELPHI2 = R(180.) / C_::PI * std::acos(COSTH4);
    R DELTHA = fd.DELTH * C_::DEG;
    R CL1 = DELPHI1 / DELTHA;
    R CL2 = DELPHI2 / DELTHA;
    // :1166-1182
    int KLP1 = KL + 1, IC = 1;
    for (int KH = 1; KH <= 2; ++KH) {
      int KLH = KL; if (KH == 2) KLH = KLP1;
      for (int Kk = 1; Kk <= KLH; ++Kk) {
        int KS = Kk; if (KH > 1) KS = KLP1 - Kk + 1;
        if (KS > KL) continue;
        R CH = R(IC) * CL1;
        JA1[(KS - 1) + KL * (KH - 1)] = JAFU(CH, Kk, KL);
        CH = R(IC) * CL2;
        JA2[(KS - 1) + KL * (KH - 1)] = JAFU(CH, Kk, KL);
      }
      IC = -1;
    }
    // :1187-1196
    CL1 = CL1 - R(int_f(CL1));
    CL2 = CL2 - R(int_f(CL2));
    ACL1 = std::fabs(CL1); ACL2 = std::fabs(CL2);
    CL11 = R(1.) - ACL1; CL21 = R(1.) - ACL2;
    R AL11 = ipow(R(1.) + ALAMD, 4), AL12 = ipow(R(1.) - ALAMD, 4);
    DAL1 = R(1.) / AL11; DAL2 = R(1.) / AL12;
    // :1201-1231
    int ISG = 1;
    for (int KH = 1; KH <= 2; ++KH) {
      R CL1H = R(ISG) * CL1, CL2H = R(ISG) * CL2;
      for (int Kk = 1; Kk <= KL; ++Kk) {
        int KS = Kk;
        if (KH == 2) KS = KL - Kk + 2;
        if (Kk == 1) KS = 1;
        int K1 = JA1[(Kk - 1) + KL * (KH - 1)];
        K1W[(KS - 1) + KL * (KH - 1)] = K1;
        int K11;
        if (CL1H < R(0.)) { K11 = K1 - 1; if (K11 < 1) K11 = KL; }
        else { K11 = K1 + 1; if (K11 > KL) K11 = 1; }
        K11W[(KS - 1) + KL * (KH - 1)] = K11;
        int K2 = JA2[(Kk - 1) + KL * (KH - 1)];
        K2W[(KS - 1) + KL * (KH - 1)] = K2;
        int K21;
        if (CL2H < R(0)) { K21 = K2 - 1; if (K21 < 1) K21 = KL; }
        else { K21 = K2 + 1; if (K21 > KL) K21 = 1; }
        K21W[(KS - 1) + KL * (KH - 1)] = K21;
      }
      ISG = -1;
    }
    // :1238-1245
    for (int M = 1; M <= ML; ++M) frlon(M) = fd.FR[M - 1];
    for (int M = 0; M >= MFRSTLW; --M) frlon(M) = frlon(M + 1) / C_::CO;
    for (int M = ML + 1; M <= ML + KFRH; ++M) frlon(M) = C_::CO * frlon(M - 1);
    // :1247-1275
    for (int M = MFRSTLW; M <= MLSTHG; ++M) {
      int i = M - MFRSTLW;
      R FRG = frlon(M);
      AF11[i] = CON * ipow(FRG, 11);
      R FLP = FRG * (R(1.) + ALAMD);
      R FLM = FRG * (R(1.) - ALAMD);
      int IKN = M + ISP;
      IKP[i] = IKN;
      R FKP = frlon(IKP[i]);
      IKP1[i] = IKP[i] + 1;
      FKLAP[i] = (FLP - FKP) / (frlon(IKP1[i]) - FKP);
      FKLAP1[i] = R(1.) - FKLAP[i];
      if (frlon(MFRSTLW) >= FLM) {
        IKM[i] = 1; IKM1[i] = 1; FKLAM[i] = R(0.); FKLAM1[i] = R(0.);
      } else {
        IKN = M + ISM;
        IKM[i] = IKN;
        R FKM = frlon(IKM[i]);
        IKM1[i] = IKM[i] + 1;
        FKLAM[i] = (FLM - FKM) / (frlon(IKM1[i]) - FKM);
        FKLAM1[i] = R(1.) - FKLAM[i];
        if (IKN < MFRSTLW) { IKM[i] = 1; FKLAM1[i] = R(0.); }
      }
    }
    // :1282-1285
    for (int I = 1; I <= KFRH; ++I) { int M = ML + I - 1; FRH[I - 1] = ipow(frlon(ML) / frlon(M), 5); }
    init_snonlin(fd);
  }

  // INIT_SNONLIN: wam_source_module.f90:1291-1523
  void init_snonlin(const FreDir<R>& fd) {
    using C_ = K<R>;
    const int ML = fd.ML;
    auto EPMMA = [](R X) { return std::exp(-std::min(R(1.25) * ipow(X, 4), R(50.))) * ipow(X, 5); };
    FTRF.assign(1 - MFRSTLW + 1, 0);
    R ALPH = R(1.) / EPMMA(R(1.));
    R FRR = R(1.);
    for (int MC = 1; MC >= MFRSTLW; --MC) { FTRF[MC - MFRSTLW] = ALPH * EPMMA(FRR); FRR = FRR * C_::CO; }
    INLCOEF.assign(5 * MLSTHG, 0); RNLCOEF.assign(25 * MLSTHG, 0);
    for (int MC = 1; MC <= MLSTHG; ++MC) {
      int MP = ikp(MC), MP1 = ikp1(MC), MM = ikm(MC), MM1 = ikm1(MC);
      R FFACP = 1, FFACP1 = 1, FFACM = 1, FFACM1 = 1, FTAIL = 1;
      int IC = MC, IP = MP, IP1 = MP1, IM = MM, IM1 = MM1;
      if (IM < 1) {
        FFACM = FTRF[IM - MFRSTLW]; IM = 1;
        if (IM1 < 1) { FFACM1 = FTRF[IM1 - MFRSTLW]; IM1 = 1; }
      }
      if (IP1 > ML) {
        int ITEMP = IP1 - ML + 1;
        if (ITEMP > (int)FRH.size()) ITEMP = (int)FRH.size();
        FFACP1 = FRH[ITEMP - 1];
        IP1 = ML;
        if (IP > ML) {
          FFACP = FRH[IP - ML + 1 - 1]; IP = ML;
          if (IC > ML) {
            FTAIL = FRH[IC - ML + 1 - 1]; IC = ML;
            if (IM1 > ML) { FFACM1 = FRH[IM1 - ML + 1 - 1]; IM1 = ML; }
          }
        }
      }
      int* ic = &INLCOEF[5 * (MC - 1)];
      ic[0] = IC; ic[1] = IP; ic[2] = IP1; ic[3] = IM; ic[4] = IM1;
      R* rc = &RNLCOEF[25 * (MC - 1)];
      int i = MC - MFRSTLW;
      R FKLAMP = FKLAP[i], FKLAMP1 = FKLAP1[i];
      R GW2 = FKLAMP1 * FFACP * DAL1;
      R GW1 = GW2 * CL11;
      GW2 = GW2 * ACL1;
      R GW4 = FKLAMP * FFACP1 * DAL1;
      R GW3 = GW4 * CL11;
      GW4 = GW4 * ACL1;
      R FKLAMPA = FKLAMP * CL11, FKLAMPB = FKLAMP * ACL1, FKLAMP2 = FKLAMP1 * ACL1;
      FKLAMP1 = FKLAMP1 * CL11;
      rc[0] = FTAIL; rc[1] = GW1; rc[2] = GW2; rc[3] = GW3; rc[4] = GW4;
      rc[5] = FKLAMPA; rc[6] = FKLAMPB; rc[7] = FKLAMP2; rc[8] = FKLAMP1;
      rc[9] = ipow(FKLAMPA, 2); rc[10] = ipow(FKLAMPB, 2); rc[11] = ipow(FKLAMP1, 2); rc[12] = ipow(FKLAMP2, 2);
      R FKLAMM = FKLAM[i], FKLAMM1 = FKLAM1[i];
      R GW6 = FKLAMM1 * FFACM * DAL2;
      R GW5 = GW6 * CL21;
      GW6 = GW6 * ACL2;
      R GW8 = FKLAMM * FFACM1 * DAL2;
      R GW7 = GW8 * CL21;
      GW8 = GW8 * ACL2;
      R FKLAMMA = FKLAMM * CL21, FKLAMMB = FKLAMM * ACL2, FKLAMM2 = FKLAMM1 * ACL2;
      FKLAMM1 = FKLAMM1 * CL21;
      rc[13] = GW5; rc[14] = GW6; rc[15] = GW7; rc[16] = GW8;
      rc[17] = FKLAMMA; rc[18] = FKLAMMB; rc[19] = FKLAMM2; rc[20] = FKLAMM1;
      rc[21] = ipow(FKLAMMA, 2); rc[22] = ipow(FKLAMMB, 2); rc[23] = ipow(FKLAMM1, 2); rc[24] = ipow(FKLAMM2, 2);
    }
  }
};

// ---- KERKEI / KZEONE: wam_source_module.f90:4058-4246 ---------------------
template <typename R> void KZEONE(R X, R Y, R& RE0, R& IM0, R& RE1, R& IM1) {
  static const R EXSQ[8] = {R(0.5641003087264E0), R(0.4120286874989E0), R(0.1584889157959E0), R(0.3078003387255E-1),
                            R(0.2778068842913E-2), R(0.1000044412325E-3), R(0.1059115547711E-5), R(0.1522475804254E-8)};
  static const R TSQ[8] = {R(0.0E0), R(3.19303633920635E-1), R(1.29075862295915E0), R(2.95837445869665E0),
                           R(5.40903159724444E0), R(8.80407957805676E0), R(1.34685357432515E1), R(2.02499163658709E1)};
  R X2, Y2, R1, R2, T1, T2, P1, P2, RTERM, ITERM, L;
  R2 = X * X + Y * Y;
  if (R2 >= R(1.96E2)) goto L50;
  if (R2 >= R(1.849E1)) goto L30;
  X2 = X / R(2.0E0); Y2 = Y / R(2.0E0);
  P1 = X2 * X2; P2 = Y2 * Y2;
  T1 = -(std::log(P1 + P2) / R(2.0E0) + R(0.5772156649015329E0));
  T2 = -std::atan2(Y, X);
  X2 = P1 - P2; Y2 = X * Y2;
  RTERM = R(1.0E0); ITERM = R(0.0E0);
  RE0 = T1; IM0 = T2;
  T1 = T1 + R(0.5E0);
  RE1 = T1; IM1 = T2;
  P2 = std::sqrt(R2);
  L = R(2.106E0) * P2 + R(4.4E0);
  if (P2 < R(8.0E-1)) L = R(2.129E0) * P2 + R(4.0E0);
  {
    int LL = nint_f(L);
    for (int N = 1; N <= LL; ++N) {
      P1 = R(N); P2 = R(N * N);
      R1 = RTERM;
      RTERM = (R1 * X2 - ITERM * Y2) / P2;
      ITERM = (R1 * Y2 + ITERM * X2) / P2;
      T1 = T1 + R(0.5E0) / P1;
      RE0 = RE0 + T1 * RTERM - T2 * ITERM;
      IM0 = IM0 + T1 * ITERM + T2 * RTERM;
      P1 = P1 + R(1.0E0);
      T1 = T1 + R(0.5E0) / P1;
      RE1 = RE1 + (T1 * RTERM - T2 * ITERM) / P1;
      IM1 = IM1 + (T1 * ITERM + T2 * RTERM) / P1;
    }
  }
  R1 = X / R2 - R(0.5E0) * (X * RE1 - Y * IM1);
  R2 = -Y / R2 - R(0.5E0) * (X * IM1 + Y * RE1);
  P1 = std::exp(X);
  RE0 = P1 * RE0; IM0 = P1 * IM0; RE1 = P1 * R1; IM1 = P1 * R2;
  return;
L30:
  X2 = R(2.0E0) * X; Y2 = R(2.0E0) * Y;
  R1 = Y2 * Y2;
  P1 = std::sqrt(X2 * X2 + R1);
  P2 = std::sqrt(P1 + X2);
  T1 = EXSQ[0] / (R(2.0E0) * P1);
  RE0 = T1 * P2; IM0 = T1 / P2;
  RE1 = R(0.0E0); IM1 = R(0.0E0);
  for (int N = 2; N <= 8; ++N) {
    T2 = X2 + TSQ[N - 1];
    P1 = std::sqrt(T2 * T2 + R1);
    P2 = std::sqrt(P1 + T2);
    T1 = EXSQ[N - 1] / P1;
    RE0 = RE0 + T1 * P2; IM0 = IM0 + T1 / P2;
    T1 = EXSQ[N - 1] * TSQ[N - 1];
    RE1 = RE1 + T1 * P2; IM1 = IM1 + T1 / P2;
  }
  T2 = -Y2 * IM0;
  RE1 = RE1 / R2;
  R2 = Y2 * IM1 / R2;
  RTERM = R(1.41421356237309E0) * std::cos(Y);
  ITERM = -R(1.41421356237309E0) * std::sin(Y);
  IM0 = RE0 * ITERM + T2 * RTERM;
  RE0 = RE0 * RTERM - T2 * ITERM;
  T1 = RE1 * RTERM - R2 * ITERM;
  T2 = RE1 * ITERM + R2 * RTERM;
  RE1 = T1 * X + T2 * Y;
  IM1 = -T1 * Y + T2 * X;
  return;
L50:
  RTERM = R(1.0E0); ITERM = R(0.0E0);
  RE0 = R(1.0E0); IM0 = R(0.0E0); RE1 = R(1.0E0); IM1 = R(0.0E0);
  P1 = R(8.0E0) * R2;
  P2 = std::sqrt(R2);
  L = R(3.91E0) + R(8.12E1) / P2;
  {
    int LL = nint_f(L);
    R1 = R(1.0E0); R2 = R(1.0E0);
    int M = -8, Kk = 3;
    for (int N = 1; N <= LL; ++N) {
      M = M + 8; Kk = Kk - M;
      R1 = R(Kk - 4) * R1;
      R2 = R(Kk) * R2;
      T1 = R(N) * P1;
      T2 = RTERM;
      RTERM = (T2 * X + ITERM * Y) / T1;
      ITERM = (-T2 * Y + ITERM * X) / T1;
      RE0 = RE0 + R1 * RTERM; IM0 = IM0 + R1 * ITERM;
      RE1 = RE1 + R2 * RTERM; IM1 = IM1 + R2 * ITERM;
    }
  }
  T1 = std::sqrt(P2 + X);
  T2 = -Y / T1;
  P1 = R(8.86226925452758E-1) / P2;
  RTERM = P1 * std::cos(Y);
  ITERM = -P1 * std::sin(Y);
  R1 = RE0 * RTERM - IM0 * ITERM;
  R2 = RE0 * ITERM + IM0 * RTERM;
  RE0 = T1 * R1 - T2 * R2;
  IM0 = T1 * R2 + T2 * R1;
  R1 = RE1 * RTERM - IM1 * ITERM;
  R2 = RE1 * ITERM + IM1 * RTERM;
  RE1 = T1 * R1 - T2 * R2;
  IM1 = T1 * R2 + T2 * R1;
}
template <typename R> void KERKEI(R X, R& KER, R& KEI) {
  R ZR = X * R(0.50) * std::sqrt(R(2.0));
  R ZI = ZR, CYR, CYI, CYR1, CYI1;
  KZEONE(ZR, ZI, CYR, CYI, CYR1, CYI1);
  KER = CYR / std::exp(ZR);
  KEI = CYI / std::exp(ZR);
}

// ---- source-term auxiliary tables ------------------------------------------
template <typename R> struct SourceTables {
  static constexpr int IAB = 200, JTOT_TAUHF = 19;
  std::vector<R> SWELLFT;            // TABU_SWELLFT :3360-3415 (1-based in reference; [i-1])
  int NSDSNTH;
  std::vector<int> INDICESSAT;       // [(k-1) + KL*(i-1)]
  std::vector<R> SATWEIGHTS;
  R X0TAUHF; std::vector<R> WTAUHF;  // INIT_X0TAUHF :3784-3849

  void build(const FreDir<R>& fd, int iphys, R ALPHA, R ZALP, R BETAMAX) {
    using C_ = K<R>;
    if (iphys == 1) {
      // TABU_SWELLFT
      SWELLFT.assign(IAB, 0);
      const int NITER = 100; const R ABMIN = R(0.3), ABMAX = R(8.0), KAPPA = R(0.40);
      R DZETA0 = R(0.0);
      R DELAB = (ABMAX - ABMIN) / R(IAB);
      R L10 = std::log(R(10.0));
      for (int I = 1; I <= IAB; ++I) {
        R ABRLOG = ABMIN + R(I) * DELAB;
        R ABR = std::exp(ABRLOG * L10);
        R FACT = R(1) / ABR / (R(21.2) * KAPPA);
        R FSUBW = R(0.05);
        for (int it = 1; it <= NITER; ++it) {
          R FSUBWMEMO = FSUBW, DZETA0MEMO = DZETA0;
          DZETA0 = FACT * std::pow(FSUBW, R(-0.5));
          R KER, KEI;
          KERKEI(R(2.0) * std::sqrt(DZETA0), KER, KEI);
          FSUBW = R(0.08) / (ipow(KER, 2) + ipow(KEI, 2));
          FSUBW = R(0.5) * (FSUBWMEMO + FSUBW);
          DZETA0 = R(0.5) * (DZETA0MEMO + DZETA0);
        }
        SWELLFT[I - 1] = FSUBW;
      }
      // INIT_SDISSP_ARD :3419-3501 (SSDSC3 = 0 so CUMULW is not built)
      const int KL = fd.KL; int KLD = KL / 2;
      NSDSNTH = std::min(nint_f(R(C_::ISDSDTH) * C_::RAD / fd.DELTH), KLD - 1);
      R DELTH_TRUNC = (fd.TH[0] + R(C_::ISDSDTH) * C_::RAD) - (fd.TH[NSDSNTH] - R(0.5) * fd.DELTH);
      DELTH_TRUNC = std::max(R(0.), std::min(DELTH_TRUNC, fd.DELTH));
      int NW = NSDSNTH * 2 + 1;
      INDICESSAT.assign(KL * NW, 0); SATWEIGHTS.assign(KL * NW, 0);
      for (int k = 1; k <= KL; ++k) {
        for (int I_INT = k - NSDSNTH; I_INT <= k + NSDSNTH; ++I_INT) {
          int J_INT = I_INT;
          if (I_INT < 1) J_INT = I_INT + KL;
          if (I_INT > KL) J_INT = I_INT - KL;
          int col = I_INT - (k - NSDSNTH) + 1;
          INDICESSAT[(k - 1) + KL * (col - 1)] = J_INT;
          R DELTH_LOC = (I_INT == k - NSDSNTH || I_INT == k + NSDSNTH) ? DELTH_TRUNC : fd.DELTH;
          SATWEIGHTS[(k - 1) + KL * (col - 1)] = DELTH_LOC * ipow(std::cos(fd.TH[k - 1] - fd.TH[J_INT - 1]), C_::ISB);
        }
      }
    } else { NSDSNTH = 0; }
    // INIT_X0TAUHF
    R X0 = R(0.005);
    for (int J = 1; J <= 30; ++J) {
      R FF = std::exp(C_::XKAPPA / (X0 + ZALP));
      R F = ALPHA * ipow(X0, 2) * FF - R(1.0);
      if (F == R(0.0)) break;
      R DF = ALPHA * FF * (R(2.0) * X0 - C_::XKAPPA * ipow(X0 / (X0 + ZALP), 2));
      X0 = X0 - F / DF;
    }
    X0TAUHF = X0;
    R CONST1 = (BETAMAX / ipow(C_::XKAPPA, 2)) / R(3.0);
    WTAUHF.assign(JTOT_TAUHF, 0);
    WTAUHF[0] = CONST1;
    for (int J = 2; J <= JTOT_TAUHF - 1; J += 2) { WTAUHF[J - 1] = R(4.0) * CONST1; WTAUHF[J] = R(2.0) * CONST1; }
    WTAUHF[JTOT_TAUHF - 1] = CONST1;
  }
};

}  // namespace wamo
