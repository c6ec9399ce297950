// Host builders of the static spectral tables consumed by the IMPLSCH and
// PROPAGS kernels.  Each builder follows the reference routine named beside
// it (myWAveModel/WAM file:line) in operation order and single-precision
// literals, because integer tables derived from floating-point expressions
// (DIA indices, frequency cut-offs, depth indices) must come out bit-exact.
// The result is a flat, reference-convention TableSet; upload.cu packs it
// into the device layout.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>
#include <string>
#include <algorithm>
#include "wamgpu_config.hpp"

namespace wamgpu {

template <typename R> R powi(R x, int n) {
  // REAL**INTEGER as the reference compiler evaluates it (binary powering).
  if (n < 0) return R(1) / powi(x, -n);
  R acc = R(1), sq = x; bool have = false;
  for (; n; n >>= 1) {
    if (n & 1) { acc = have ? acc * sq : sq; have = true; }
    if (n > 1) sq = sq * sq;
  }
  return acc;
}
inline int f_nint(double x) { return (int)std::lround(x); }
inline int f_int(double x) { return (int)std::trunc(x); }

template <typename R> struct Phys {
  static constexpr R G = R(9.806), PI = R(3.1415927), ZPI = R(2.) * PI, DEG = R(180.) / PI, RAD = PI / R(180.);
  static constexpr R CIRC = R(40000000.), RE = CIRC / ZPI, ROAIR = R(1.225), RNUAIR = R(1.5E-5),
                     RNUAIRM = R(0.11) * RNUAIR, ROWATER = R(1000.), XKAPPA = R(0.40), XNLEV = R(10.0), DKMAX = R(40.);
  static constexpr R CO = R(1.1);
};

// Dispersion solver AKI (wam_general_module.f90:301-364).
template <typename R> R aki(R om, R depth) {
  using P = Phys<R>;
  R k = std::max(powi(om, 2) / (R(4.) * P::G), om / (R(2.) * std::sqrt(P::G * depth)));
  R kprev = R(10000.);
  while (std::fabs(kprev - k) > R(0.0001) * k) {
    R bo = depth * k;
    if (bo > P::DKMAX) { k = powi(om, 2) / P::G; break; }
    kprev = k;
    R th = (P::G * k) * std::tanh(bo);
    R sth = std::sqrt(th);
    k = k + (om - sth) * sth * R(2.) / (th / k + P::G * bo / powi(std::cosh(bo), 2));
  }
  return k;
}

// Finite-depth SNL scaling TRANSF (wam_interface_module.f90:2614-2680).
template <typename R> R transf(R xk, R d) {
  using P = Phys<R>;
  if (!(d < R(999.) && d > R(0.))) return R(1.);
  R x = xk * d;
  if (x > P::DKMAX) return R(1.);
  R t0 = std::tanh(x), om = std::sqrt((P::G * xk) * t0), c0 = om / xk;
  R vg = (x < R(0.0001)) ? c0 : (R(0.5) * c0) * (R(1.) + R(2.) * x / std::sinh(R(2.) * x));
  R t2 = powi(t0, 2);
  R dvg = powi(t0 - x * (R(1.) - t2), 2) + ((R(4.) * powi(x, 2)) * t2) * (R(1.) - t2);
  R xnl1 = ((R(9.) * powi(t0, 4) - R(10.) * t2) + R(9.)) / (R(8.) * powi(t0, 3));
  R xnl2 = (powi(R(2.) * vg - R(0.5) * c0, 2) / (P::G * d - powi(vg, 2)) + R(1.)) / x;
  return powi(xnl1 - xnl2, 2) / (dvg * powi(t0, 8));
}

// Modified Bessel functions of complex argument (wam_source_module.f90:4080-4246)
template <typename R> static void kzeone(R x, R y, R& re0, R& im0, R& re1, R& im1) {
  const R exsq[8] = {R(0.5641003087264E0), R(0.4120286874989E0), R(0.1584889157959E0), R(0.3078003387255E-1),
                     R(0.2778068842913E-2), R(0.1000044412325E-3), R(0.1059115547711E-5), R(0.1522475804254E-8)};
  const R tsq[8] = {R(0.0E0), R(3.19303633920635E-1), R(1.29075862295915E0), R(2.95837445869665E0),
                    R(5.40903159724444E0), R(8.80407957805676E0), R(1.34685357432515E1), R(2.02499163658709E1)};
  R r2 = x * x + y * y;
  if (r2 < R(1.849E1)) {  // power series
    R x2 = x / R(2.0E0), y2 = y / R(2.0E0), p1 = x2 * x2, p2 = y2 * y2;
    R t1 = -(std::log(p1 + p2) / R(2.0E0) + R(0.5772156649015329E0));
    R t2 = -std::atan2(y, x);
    x2 = p1 - p2; y2 = x * y2;
    R rt = R(1.0E0), it = R(0.0E0);
    re0 = t1; im0 = t2; t1 = t1 + R(0.5E0); re1 = t1; im1 = t2;
    p2 = std::sqrt(r2);
    R l = (p2 < R(8.0E-1)) ? R(2.129E0) * p2 + R(4.0E0) : R(2.106E0) * p2 + R(4.4E0);
    int ll = f_nint(l);
    for (int n = 1; n <= ll; ++n) {
      p1 = R(n); p2 = R(n * n);
      R r1 = rt;
      rt = (r1 * x2 - it * y2) / p2;
      it = (r1 * y2 + it * x2) / p2;
      t1 = t1 + R(0.5E0) / p1;
      re0 = re0 + t1 * rt - t2 * it; im0 = im0 + t1 * it + t2 * rt;
      p1 = p1 + R(1.0E0);
      t1 = t1 + R(0.5E0) / p1;
      re1 = re1 + (t1 * rt - t2 * it) / p1; im1 = im1 + (t1 * it + t2 * rt) / p1;
    }
    R r1 = x / r2 - R(0.5E0) * (x * re1 - y * im1);
    R rr2 = -y / r2 - R(0.5E0) * (x * im1 + y * re1);
    p1 = std::exp(x);
    re0 = p1 * re0; im0 = p1 * im0; re1 = p1 * r1; im1 = p1 * rr2;
  } else if (r2 < R(1.96E2)) {  // Gauss-Hermite quadrature
    R x2 = R(2.0E0) * x, y2 = R(2.0E0) * y, r1 = y2 * y2;
    R p1 = std::sqrt(x2 * x2 + r1), p2 = std::sqrt(p1 + x2), t1 = exsq[0] / (R(2.0E0) * p1);
    re0 = t1 * p2; im0 = t1 / p2; re1 = R(0.0E0); im1 = R(0.0E0);
    for (int n = 1; n < 8; ++n) {
      R t2 = x2 + tsq[n];
      p1 = std::sqrt(t2 * t2 + r1); p2 = std::sqrt(p1 + t2);
      t1 = exsq[n] / p1;
      re0 = re0 + t1 * p2; im0 = im0 + t1 / p2;
      t1 = exsq[n] * tsq[n];
      re1 = re1 + t1 * p2; im1 = im1 + t1 / p2;
    }
    R t2 = -y2 * im0;
    re1 = re1 / r2;
    R rr2 = y2 * im1 / r2;
    R rt = R(1.41421356237309E0) * std::cos(y), it = -R(1.41421356237309E0) * std::sin(y);
    im0 = re0 * it + t2 * rt;
    re0 = re0 * rt - t2 * it;
    t1 = re1 * rt - rr2 * it;
    t2 = re1 * it + rr2 * rt;
    re1 = t1 * x + t2 * y;
    im1 = -t1 * y + t2 * x;
  } else {  // asymptotic expansion
    R rt = R(1.0E0), it = R(0.0E0);
    re0 = R(1.0E0); im0 = R(0.0E0); re1 = R(1.0E0); im1 = R(0.0E0);
    R p1 = R(8.0E0) * r2, p2 = std::sqrt(r2);
    int ll = f_nint(R(3.91E0) + R(8.12E1) / p2);
    R r1 = R(1.0E0), rr2 = R(1.0E0);
    int mm = -8, kk = 3;
    for (int n = 1; n <= ll; ++n) {
      mm = mm + 8; kk = kk - mm;
      r1 = R(kk - 4) * r1; rr2 = R(kk) * rr2;
      R t1 = R(n) * p1, t2 = rt;
      rt = (t2 * x + it * y) / t1;
      it = (-t2 * y + it * x) / t1;
      re0 = re0 + r1 * rt; im0 = im0 + r1 * it;
      re1 = re1 + rr2 * rt; im1 = im1 + rr2 * it;
    }
    R t1 = std::sqrt(p2 + x), t2 = -y / t1;
    p1 = R(8.86226925452758E-1) / p2;
    rt = p1 * std::cos(y); it = -p1 * std::sin(y);
    r1 = re0 * rt - im0 * it; rr2 = re0 * it + im0 * rt;
    re0 = t1 * r1 - t2 * rr2; im0 = t1 * rr2 + t2 * r1;
    r1 = re1 * rt - im1 * it; rr2 = re1 * it + im1 * rt;
    re1 = t1 * r1 - t2 * rr2; im1 = t1 * rr2 + t2 * r1;
  }
}

// All static tables of one configuration, reference conventions (1-based
// index values, 0 = not used).  Frequency-dependent DIA arrays span
// M = MFRSTLW..MLSTHG and are stored at [M - MFRSTLW].
template <typename R> struct TableSet {
  int KL = 0, ML = 0;
  // wam_fre_dir_module.f90:297-459
  std::vector<R> FR, DF, DFIM, DFIMOFR, FR5, FRM5, RHOWG_DFIM, GOM, C, TH, COSTH, SINTH;
  std::vector<R> DFIM_FR, DFIM_FR2;  // DF*FR*DELTH, DF*FR**2*DELTH (fre_dir:392-393)
  R DELTH = 0, DELTR = 0, INV_LOG_CO = 0, MO_TAIL = 0, MM1_TAIL = 0, MP1_TAIL = 0, MP2_TAIL = 0;
  // wam_tables_module.f90:388-464 ([(jd-1) + NDEPTH*m])
  int NDEPTH = 0; R DEPTHA = 0, DEPTHD = 0;
  std::vector<R> TFAK, TCGOND, TSIHKD;
  // wam_tables_module.f90:315-384 ([(ju-1) + JUMAX*m])
  static constexpr int JUMAX = 300;
  R DELU = 0; std::vector<R> FLMINFR;
  // wam_source_module.f90:1056-1523
  int MFRSTLW = 0, MLSTHG = 0, KFRH = 0;
  R ACL1 = 0, ACL2 = 0, CL11 = 0, CL21 = 0, DAL1 = 0, DAL2 = 0;
  std::vector<int> IKP, IKP1, IKM, IKM1, K1W, K2W, K11W, K21W, INLCOEF;
  std::vector<R> AF11, FKLAP, FKLAP1, FKLAM, FKLAM1, FRH, RNLCOEF;
  // wam_source_module.f90:3360-3565, 3784-3849
  std::vector<R> SWELLFT, SATWEIGHTS, WTAUHF;
  std::vector<int> INDICESSAT;
  int NSDSNTH = 0;
  R X0TAUHF = 0;

  void build(const Config& c) {
    build_fre_dir(c);
    build_shallow(c);
    build_min_energy(c);
    build_dia();
    build_source_aux(c);
  }

  void build_fre_dir(const Config& c) {
    using P = Phys<R>;
    KL = c.kl; ML = c.ml;
    FR.resize(ML);
    FR[0] = powi(P::CO, -c.iref + 1) * R(c.fr1);
    INV_LOG_CO = R(1.) / std::log10(P::CO);
    for (int m = 1; m < ML; ++m) FR[m] = P::CO * FR[m - 1];
    FR5.resize(ML); FRM5.resize(ML); GOM.resize(ML); C.resize(ML);
    for (int m = 0; m < ML; ++m) {
      FR5[m] = powi(FR[m], 5);
      FRM5[m] = R(1) / FR5[m];
      GOM[m] = P::G / ((R(2.) * P::ZPI) * FR[m]);
      C[m] = P::G / (P::ZPI * FR[m]);
    }
    DELTH = P::ZPI / R(KL);
    DELTR = DELTH * P::RE;
    TH.resize(KL); COSTH.resize(KL); SINTH.resize(KL);
    for (int k = 0; k < KL; ++k) {
      TH[k] = R(k) * DELTH + R(0.5) * DELTH;
      COSTH[k] = std::cos(TH[k]);
      SINTH[k] = std::sin(TH[k]);
    }
    const R co1 = R(0.5) * (P::CO - R(1.));
    DF.resize(ML);
    for (int m = 0; m < ML; ++m) DF[m] = (m == 0) ? co1 * FR[0] : (m == ML - 1 ? co1 * FR[ML - 2] : co1 * (FR[m] + FR[m - 1]));
    DFIM.resize(ML); DFIMOFR.resize(ML); RHOWG_DFIM.resize(ML);
    const R rowg = P::ROWATER * P::G;
    for (int m = 0; m < ML; ++m) {
      DFIM[m] = DF[m] * DELTH;
      DFIMOFR[m] = DFIM[m] / FR[m];
      RHOWG_DFIM[m] = ((rowg * DELTH) * std::log(P::CO)) * FR[m];
    }
    RHOWG_DFIM[0] = R(0.5) * RHOWG_DFIM[0];
    RHOWG_DFIM[ML - 1] = R(0.5) * RHOWG_DFIM[ML - 1];
    const int ex_tail = -5;
    MO_TAIL = -(DELTH / R(ex_tail + 1) * FR[ML - 1]);
    MM1_TAIL = -(DELTH / R(ex_tail));
    MP1_TAIL = -(DELTH / R(ex_tail + 2) * powi(FR[ML - 1], 2));
    MP2_TAIL = -(DELTH / R(ex_tail + 3) * powi(FR[ML - 1], 3));
    DFIM_FR.resize(ML); DFIM_FR2.resize(ML);
    for (int m = 0; m < ML; ++m) {
      const R df_fr = DF[m] * FR[m], df_fr2 = df_fr * FR[m];
      DFIM_FR[m] = df_fr * DELTH;
      DFIM_FR2[m] = df_fr2 * DELTH;
    }
  }

  void build_shallow(const Config& c) {
    using P = Phys<R>;
    NDEPTH = c.ndepth; DEPTHA = R(c.deptha); DEPTHD = R(c.depthd);
    TFAK.assign((size_t)NDEPTH * ML, 0); TCGOND = TFAK; TSIHKD = TFAK;
    const R gh = P::G / (R(4.) * P::PI);
    for (int m = 0; m < ML; ++m) {
      R om = P::ZPI * FR[m];
      for (int jd = 0; jd < NDEPTH; ++jd) {
        R ad = DEPTHA * powi(DEPTHD, jd);
        R ak = aki(om, ad), akd = ak * ad;
        size_t i = jd + (size_t)NDEPTH * m;
        TFAK[i] = ak;
        if (akd <= R(10.0)) {
          TCGOND[i] = R(0.5) * std::sqrt(P::G * std::tanh(akd) / ak) * (R(1.0) + R(2.0) * akd / std::sinh(R(2.) * akd));
          TSIHKD[i] = om / std::sinh(R(2.) * akd);
        } else {
          TCGOND[i] = gh / FR[m];
          TSIHKD[i] = R(0.);
        }
      }
    }
  }

  void build_min_energy(const Config& c) {
    // MIN_ENERGY with FETCH_LAW and JONSWAP (wam_jonswap_module.f90:63-211)
    using P = Phys<R>;
    DELU = R(75.) / R(JUMAX);
    R fetch = std::min(R(0.5) * R(c.delphi), R(25000.));
    R fpmax = FR[ML - 1];
    std::vector<R> alph(JUMAX), fp(JUMAX);
    const R A = R(2.84), D = -(R(3.) / R(10.)), B = R(0.033), E = R(2.) / R(3.);
    for (int j = 0; j < JUMAX; ++j) {
      R u = R(j + 1) * DELU;
      if (u > R(0.1E-08)) {
        R ug = P::G / u;
        R f = std::max(R(0.13), A * std::pow((P::G * fetch) / powi(u, 2), D));
        f = std::min(f, fpmax / ug);
        alph[j] = std::max(R(0.0081), B * std::pow(f, E));
        fp[j] = f * ug;
      } else { alph[j] = R(0.0081); fp[j] = fpmax; }
      alph[j] = R(0.01) * alph[j];
    }
    FLMINFR.assign((size_t)JUMAX * ML, 0);
    const R g2zpi4 = powi(P::G, 2) / powi(P::ZPI, 4);
    const R loggam = std::log(R(3.000000));
    const R saa = R(0.5) / (R(7.000000E-02) * R(7.000000E-02)), sbb = R(0.5) / (R(9.000000E-02) * R(9.000000E-02));
    for (int m = 0; m < ML; ++m) {
      R f = FR[m], g2 = g2zpi4 * powi(f, -5);
      for (int j = 0; j < JUMAX; ++j) {
        R arg = R(1.25) * powi(fp[j] / f, 4), et = R(0.);
        if (arg < R(50.)) {
          et = alph[j] * g2 * std::exp(-arg);
          arg = (f > fp[j]) ? sbb * powi(f / fp[j] - R(1.), 2) : saa * powi(f / fp[j] - R(1.), 2);
          if (arg < R(99.)) et = et * std::exp(loggam * std::exp(-arg));
        }
        FLMINFR[j + (size_t)JUMAX * m] = std::max(et, R(0.000001));
      }
    }
  }

  void build_dia() {
    using P = Phys<R>;
    const R lam = R(0.25), con = R(3000.);
    R f1p1 = std::log10(P::CO);
    int isp = f_int(std::log10(R(1.) + lam) / f1p1 + R(.000001));
    int ism = (int)std::floor(std::log10(R(1.) - lam) / f1p1 + R(.0000001));
    MFRSTLW = 1 + ism; MLSTHG = ML - ism; KFRH = -ism + isp + 2;
    // angular geometry of the quadruplet (NLWEIGT :1153-1161)
    R xf = powi((R(1.) + lam) / (R(1.) - lam), 4);
    R costh3 = (R(1.) + R(2.) * lam + R(2.) * powi(lam, 3)) / powi(R(1.) + lam, 2);
    R delphi1 = -(R(180.) / P::PI * std::acos(costh3));
    R costh4 = std::sqrt(R(1.) - xf + xf * powi(costh3, 2));
    R delphi2 = R(180.) / P::PI * std::acos(costh4);
    R deltha = DELTH * P::DEG;
    R cl1 = delphi1 / deltha, cl2 = delphi2 / deltha;
    // JA1/JA2 through JAFU (src/chief/jafu.f90:3-39)
    auto jafu = [&](R cl, int j) { int r = j + f_int(cl); if (r <= 0) r += KL; if (r > KL) r -= KL; return r; };
    std::vector<int> ja1(2 * KL), ja2(2 * KL);
    for (int kh = 1; kh <= 2; ++kh) {
      int sgn = (kh == 1) ? 1 : -1, klh = (kh == 1) ? KL : KL + 1;
      for (int k = 1; k <= klh; ++k) {
        int ks = (kh > 1) ? KL + 2 - k : k;
        if (ks > KL) continue;
        ja1[(ks - 1) + KL * (kh - 1)] = jafu(R(sgn) * cl1, k);
        ja2[(ks - 1) + KL * (kh - 1)] = jafu(R(sgn) * cl2, k);
      }
    }
    cl1 = cl1 - R(f_int(cl1));
    cl2 = cl2 - R(f_int(cl2));
    ACL1 = std::fabs(cl1); ACL2 = std::fabs(cl2);
    CL11 = R(1.) - ACL1; CL21 = R(1.) - ACL2;
    DAL1 = R(1.) / powi(R(1.) + lam, 4);
    DAL2 = R(1.) / powi(R(1.) - lam, 4);
    K1W.assign(2 * KL, 0); K2W = K1W; K11W = K1W; K21W = K1W;
    for (int kh = 1; kh <= 2; ++kh) {
      R sg = (kh == 1) ? R(1) : R(-1);
      R c1h = sg * cl1, c2h = sg * cl2;
      for (int k = 1; k <= KL; ++k) {
        int ks = (k == 1) ? 1 : (kh == 2 ? KL - k + 2 : k);
        int slot = (ks - 1) + KL * (kh - 1);
        int k1 = ja1[(k - 1) + KL * (kh - 1)], k2 = ja2[(k - 1) + KL * (kh - 1)];
        K1W[slot] = k1;
        K11W[slot] = (c1h < R(0.)) ? (k1 - 1 < 1 ? KL : k1 - 1) : (k1 + 1 > KL ? 1 : k1 + 1);
        K2W[slot] = k2;
        K21W[slot] = (c2h < R(0)) ? (k2 - 1 < 1 ? KL : k2 - 1) : (k2 + 1 > KL ? 1 : k2 + 1);
      }
    }
    // extended frequency axis and the interpolation weights (:1238-1285)
    auto idx = [&](int m) { return m - MFRSTLW; };
    std::vector<R> frl(ML + KFRH - MFRSTLW + 1);
    for (int m = 1; m <= ML; ++m) frl[idx(m)] = FR[m - 1];
    for (int m = 0; m >= MFRSTLW; --m) frl[idx(m)] = frl[idx(m + 1)] / P::CO;
    for (int m = ML + 1; m <= ML + KFRH; ++m) frl[idx(m)] = P::CO * frl[idx(m - 1)];
    int n = MLSTHG - MFRSTLW + 1;
    IKP.assign(n, 0); IKP1 = IKP; IKM = IKP; IKM1 = IKP;
    AF11.assign(n, 0); FKLAP = AF11; FKLAP1 = AF11; FKLAM = AF11; FKLAM1 = AF11;
    for (int m = MFRSTLW; m <= MLSTHG; ++m) {
      int i = idx(m);
      R frg = frl[i];
      AF11[i] = con * powi(frg, 11);
      R flp = frg * (R(1.) + lam), flm = frg * (R(1.) - lam);
      IKP[i] = m + isp;
      R fkp = frl[idx(IKP[i])];
      IKP1[i] = IKP[i] + 1;
      FKLAP[i] = (flp - fkp) / (frl[idx(IKP1[i])] - fkp);
      FKLAP1[i] = R(1.) - FKLAP[i];
      if (frl[idx(MFRSTLW)] >= flm) {
        IKM[i] = 1; IKM1[i] = 1; FKLAM[i] = R(0.); FKLAM1[i] = R(0.);
      } else {
        int ikn = m + ism;
        IKM[i] = ikn;
        R fkm = frl[idx(ikn)];
        IKM1[i] = ikn + 1;
        FKLAM[i] = (flm - fkm) / (frl[idx(IKM1[i])] - fkm);
        FKLAM1[i] = R(1.) - FKLAM[i];
        if (ikn < MFRSTLW) { IKM[i] = 1; FKLAM1[i] = R(0.); }
      }
    }
    FRH.assign(KFRH, 0);
    for (int i = 0; i < KFRH; ++i) FRH[i] = powi(frl[idx(ML)] / frl[idx(ML + i)], 5);
    // INIT_SNONLIN (:1291-1523): folded indices and weights per frequency MC
    auto epmma = [](R x) { return std::exp(-std::min(R(1.25) * powi(x, 4), R(50.))) * powi(x, 5); };
    std::vector<R> ftrf(2 - MFRSTLW);
    R alph = R(1.) / epmma(R(1.)), frr = R(1.);
    for (int mc = 1; mc >= MFRSTLW; --mc) { ftrf[mc - MFRSTLW] = alph * epmma(frr); frr = frr * P::CO; }
    INLCOEF.assign(5 * MLSTHG, 0); RNLCOEF.assign(25 * MLSTHG, 0);
    for (int mc = 1; mc <= MLSTHG; ++mc) {
      int i = idx(mc);
      R ffacp = 1, ffacp1 = 1, ffacm = 1, ffacm1 = 1, ftail = 1;
      int ic = mc, ip = IKP[i], ip1 = IKP1[i], im = IKM[i], im1 = IKM1[i];
      if (im < 1) {
        ffacm = ftrf[im - MFRSTLW]; im = 1;
        if (im1 < 1) { ffacm1 = ftrf[im1 - MFRSTLW]; im1 = 1; }
      }
      if (ip1 > ML) {
        ffacp1 = FRH[std::min(ip1 - ML + 1, KFRH) - 1];
        ip1 = ML;
        if (ip > ML) {
          ffacp = FRH[ip - ML]; ip = ML;
          if (ic > ML) {
            ftail = FRH[ic - ML]; ic = ML;
            if (im1 > ML) { ffacm1 = FRH[im1 - ML]; im1 = ML; }
          }
        }
      }
      int* ii = &INLCOEF[5 * (mc - 1)];
      ii[0] = ic; ii[1] = ip; ii[2] = ip1; ii[3] = im; ii[4] = im1;
      R* rc = &RNLCOEF[25 * (mc - 1)];
      R wp = FKLAP[i], wp1 = FKLAP1[i];
      R gw2 = wp1 * ffacp * DAL1, gw4 = wp * ffacp1 * DAL1;
      R pa = wp * CL11, pb = wp * ACL1, p2 = wp1 * ACL1, p1 = wp1 * CL11;
      rc[0] = ftail; rc[1] = gw2 * CL11; rc[2] = gw2 * ACL1; rc[3] = gw4 * CL11; rc[4] = gw4 * ACL1;
      rc[5] = pa; rc[6] = pb; rc[7] = p2; rc[8] = p1;
      rc[9] = powi(pa, 2); rc[10] = powi(pb, 2); rc[11] = powi(p1, 2); rc[12] = powi(p2, 2);
      R wm = FKLAM[i], wm1 = FKLAM1[i];
      R gw6 = wm1 * ffacm * DAL2, gw8 = wm * ffacm1 * DAL2;
      R ma = wm * CL21, mb = wm * ACL2, m2 = wm1 * ACL2, m1 = wm1 * CL21;
      rc[13] = gw6 * CL21; rc[14] = gw6 * ACL2; rc[15] = gw8 * CL21; rc[16] = gw8 * ACL2;
      rc[17] = ma; rc[18] = mb; rc[19] = m2; rc[20] = m1;
      rc[21] = powi(ma, 2); rc[22] = powi(mb, 2); rc[23] = powi(m1, 2); rc[24] = powi(m2, 2);
    }
  }

  void build_source_aux(const Config& c) {
    using P = Phys<R>;
    const R alpha = R(c.alpha), zalp = R(c.zalp), betamax = R(c.betamax);
    SWELLFT.clear(); SATWEIGHTS.clear(); INDICESSAT.clear(); NSDSNTH = 0;
    if (c.iphys == 1) {
      // TABU_SWELLFT (:3360-3415): friction factor of the oscillatory boundary layer
      const int iab = 200;
      SWELLFT.assign(iab, 0);
      const R abmin = R(0.3), delab = (R(8.0) - abmin) / R(iab), l10 = std::log(R(10.0));
      R dzeta0 = R(0.0);
      for (int i = 1; i <= iab; ++i) {
        R abr = std::exp((abmin + R(i) * delab) * l10);
        R fact = R(1) / abr / (R(21.2) * R(0.40));
        R fsubw = R(0.05);
        for (int it = 0; it < 100; ++it) {
          R fsubw_old = fsubw, dzeta_old = dzeta0;
          dzeta0 = fact * std::pow(fsubw, R(-0.5));
          R zr = R(2.0) * std::sqrt(dzeta0) * R(0.50) * std::sqrt(R(2.0));
          R cyr, cyi, cyr1, cyi1;
          kzeone(zr, zr, cyr, cyi, cyr1, cyi1);
          R ker = cyr / std::exp(zr), kei = cyi / std::exp(zr);
          fsubw = R(0.08) / (powi(ker, 2) + powi(kei, 2));
          fsubw = R(0.5) * (fsubw_old + fsubw);
          dzeta0 = R(0.5) * (dzeta_old + dzeta0);
        }
        SWELLFT[i - 1] = fsubw;
      }
      // INIT_SDISSP_ARD (:3419-3501): directional smoothing of the saturation spectrum
      int kld = KL / 2;
      NSDSNTH = std::min(f_nint(R(80) * P::RAD / DELTH), kld - 1);
      R trunc = (TH[0] + R(80) * P::RAD) - (TH[NSDSNTH] - R(0.5) * DELTH);
      trunc = std::max(R(0.), std::min(trunc, DELTH));
      int nw = 2 * NSDSNTH + 1;
      INDICESSAT.assign(KL * nw, 0); SATWEIGHTS.assign(KL * nw, 0);
      for (int k = 1; k <= KL; ++k)
        for (int j = 0; j < nw; ++j) {
          int ii = k - NSDSNTH + j, jj = ii < 1 ? ii + KL : (ii > KL ? ii - KL : ii);
          INDICESSAT[(k - 1) + KL * j] = jj;
          R dl = (j == 0 || j == nw - 1) ? trunc : DELTH;
          SATWEIGHTS[(k - 1) + KL * j] = dl * powi(std::cos(TH[k - 1] - TH[jj - 1]), 2);
        }
    }
    // INIT_X0TAUHF (:3784-3849)
    R x0 = R(0.005);
    for (int j = 0; j < 30; ++j) {
      R ff = std::exp(P::XKAPPA / (x0 + zalp));
      R f = alpha * powi(x0, 2) * ff - R(1.0);
      if (f == R(0.0)) break;
      R df = alpha * ff * (R(2.0) * x0 - P::XKAPPA * powi(x0 / (x0 + zalp), 2));
      x0 = x0 - f / df;
    }
    X0TAUHF = x0;
    R c1 = (betamax / powi(P::XKAPPA, 2)) / R(3.0);
    WTAUHF.assign(19, R(0));
    for (int j = 0; j < 19; ++j) WTAUHF[j] = (j == 0 || j == 18) ? c1 : ((j % 2 == 1) ? R(4.0) * c1 : R(2.0) * c1);
  }
};

}  // namespace wamgpu
