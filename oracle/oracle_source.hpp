// ORACLE — test infrastructure only (see oracle_tables.hpp header).
//
// Statement-order restatement of IMPLSCH (wam_source_module.f90:374-700) and
// its ST4 (IPHYS=1) and ST6 (IPHYS=2) callees.  The reference loops over a
// slab of sea points with IJ innermost; every operation of one point depends
// only on that point's data (STRESSO's MAXVAL(MIJ) bound only adds exact
// zeros), so this restatement runs the same per-point statement sequence one
// point at a time.  Per point the spectrum is F[k + KL*m] (k, m 0-based).
#pragma once
#include "oracle_tables.hpp"

namespace wamo {

template <typename R> struct SourceModel {
  using C_ = K<R>;
  OracleConfig cfg;
  const FreDir<R>* fd; const ShallowTables<R>* sh; const MinEnergy<R>* me;
  const DiaTables<R>* dia; const SourceTables<R>* st;
  R BETAMAX, ZALP, ALPHA, TAUWSHELTER, CDFAC;
  std::vector<R> ENH_table;  // MAKE_SHALLOW_SNL table [(ij) + nsea*(mc-1)] when ISNONLIN != 0
  int enh_nsea = 0;

  int KL() const { return fd->KL; }
  int ML() const { return fd->ML; }

  // ---- spectral integrals: wam_interface_module.f90 -----------------------
  // TOTAL_ENERGY_B :1342-1410
  R total_energy(const R* F, const uint8_t* mask) const {
    int kl = KL(), ml = ML();
    std::vector<R> temp(ml);
    for (int m = 0; m < ml; ++m) {
      R s = R(0);
      for (int k = 0; k < kl; ++k) if (!mask || mask[k + kl * m]) s = s + F[k + kl * m];
      temp[m] = s;
    }
    R e = fd->MO_TAIL * temp[ml - 1];
    for (int m = 0; m < ml; ++m) e = e + temp[m] * fd->DFIM[m];
    return std::max(e, C_::EMIN);
  }
  // FEMEAN :207-286
  R femean(const R* F, R emean, const uint8_t* mask) const {
    int kl = KL(), ml = ML();
    std::vector<R> temp(ml);
    for (int m = 0; m < ml; ++m) {
      R s = R(0);
      for (int k = 0; k < kl; ++k) if (!mask || mask[k + kl * m]) s = s + F[k + kl * m];
      temp[m] = s;
    }
    R fm = fd->MM1_TAIL * temp[ml - 1];
    for (int m = 0; m < ml; ++m) fm = fm + temp[m] * fd->DFIMOFR[m];
    return emean / std::max(fm, C_::EMIN);
  }
  // WM1_WM2_WAVENUMBER_B :1591-1716, WM1 only (AKMEAN)
  R wm1(const R* F, R emean, int indep) const {
    int kl = KL(), ml = ML();
    std::vector<R> temp(ml);
    for (int m = 0; m < ml; ++m) { R s = 0; for (int k = 0; k < kl; ++k) s = s + F[k + kl * m]; temp[m] = s; }
    R DEL2 = std::sqrt(C_::G) / C_::ZPI;
    R w = fd->MM1_TAIL * DEL2 * temp[ml - 1];
    if (cfg.shallow_run) {
      for (int m = 0; m < ml; ++m) w = w + temp[m] / std::sqrt(sh->tfak(indep, m)) * fd->DFIM[m];
    } else {
      for (int m = 0; m < ml; ++m) w = w + temp[m] * fd->DFIMOFR[m] * DEL2;
    }
    if (emean > C_::EMIN) return ipow(emean / w, 2);
    return R(1.);
  }

  // ---- AIRSEA :868-971 ------------------------------------------------------
  void airsea(R UTOP, R TAUW, R& USTAR, R& Z0) const {
    const int NITER = 15; const R TWOXMP1 = R(3.0), EPSUS = R(1.0E-6), ACD = R(8.0E-4), BCD = R(8.0E-5);
    R XLOGXL = std::log(C_::XNLEV);
    R ALPHAOG = ALPHA / C_::G;
    R XKUTOP = C_::XKAPPA * UTOP;
    R USTOLD = UTOP * std::sqrt(ACD + BCD * UTOP);
    R TAUOLD = std::max(ipow(USTOLD, 2), TAUW + C_::EPS1);
    USTAR = std::sqrt(TAUOLD);
    R USTM1 = R(1.0) / std::max(USTAR, EPSUS);
    R Z0CH = 0;
    for (int it = 1; it <= NITER; ++it) {
      R X = TAUW / TAUOLD;
      Z0CH = ALPHAOG * TAUOLD / std::sqrt(std::max(R(1.0) - X, C_::EPS1));
      R Z0VIS = C_::RNUAIRM * USTM1;
      R Z0TOT = Z0CH + Z0VIS;
      R XOLOGZ0 = R(1.0) / (XLOGXL - std::log(Z0TOT));
      R Fv = USTAR - XKUTOP * XOLOGZ0;
      R ZZ = USTM1 * (Z0CH * (R(2.0) - TWOXMP1 * X) / (R(1.0) - X) - Z0VIS) / Z0TOT;
      R DELF = R(1.0) - XKUTOP * ipow(XOLOGZ0, 2) * ZZ;
      USTAR = USTAR - Fv / DELF;
      R TAUNEW = std::max(ipow(USTAR, 2), TAUW + C_::EPS1);
      USTAR = std::sqrt(TAUNEW);
      if (TAUNEW == TAUOLD) break;
      USTM1 = R(1.0) / std::max(USTAR, EPSUS);
      TAUOLD = TAUNEW;
    }
    Z0 = Z0CH;
  }

  // ---- W3FLX4 :5372-5443 ----------------------------------------------------
  void w3flx4(R U10, R& UST, R& Z0, R& CD) const {
    R FLX4A0 = CDFAC;
    if (U10 >= R(50.33)) { UST = R(2.026) * std::sqrt(FLX4A0); CD = ipow(UST / U10, 2); }
    else {
      CD = FLX4A0 * (R(8.058) + R(0.967) * U10 - R(0.016) * ipow(U10, 2)) * R(1E-4);
      UST = U10 * std::sqrt(CD);
    }
    Z0 = C_::XNLEV * std::exp(-R(0.4) / std::sqrt(CD));
  }

  // ---- WSIGSTAR :4250-4339 --------------------------------------------------
  R wsigstar(R USTAR, R Z0, R WSTAR) const {
    const R WSPMIN = R(1.0), BG_GUST = R(0.0), ONETHIRD = R(1.0) / R(3.0), LOG10_ = std::log(R(10.0));
    const R C1 = R(1.03E-3), C2 = R(0.04E-3), P1 = R(1.48), P2 = R(-0.21);
    R XKAPPAD = R(1.0) / C_::XKAPPA;
    R U10 = USTAR * XKAPPAD * (LOG10_ - std::log(Z0));
    U10 = std::max(U10, WSPMIN);
    R U10M1 = R(1.0) / U10;
    R C2U10P1 = C2 * std::pow(U10, P1);
    R U10P2 = std::pow(U10, P2);
    R C_D = (C1 + C2U10P1) * U10P2;
    R DC_DDU = (P2 * C1 + (P1 + P2) * C2U10P1) * U10P2 * U10M1;
    R SIG_CONV = R(1.0) + R(0.5) * U10 / C_D * DC_DDU;
    return std::min(R(0.1), SIG_CONV * U10M1 *
                                std::pow(BG_GUST * ipow(USTAR, 3) + R(0.5) * C_::XKAPPA * ipow(WSTAR, 3), ONETHIRD));
  }

  // ---- SINPUT_ARD :2312-2738 ------------------------------------------------
  void sinput_ard(const R* F, R* SL, R* SPOS, R* FL, R USTAR, R UDIR, R Z0, R ROAIRN, R WSTAR, int INDEP,
                  uint8_t* LLWS) const {
    const int kl = KL(), ml = ML(), NGST = 2, IAB = SourceTables<R>::IAB;
    const R SWELLF = R(0.66), SWELLF2 = R(-0.018), SWELLF3 = R(0.022), SWELLF4 = R(1.5E05), SWELLF5 = R(1.2),
            SWELLF7 = R(3.6E05), Z0RAT = R(0.04), Z0TUBMAX = R(0.0005), ABMIN = R(0.3), ABMAX = R(8.0);
    R ROG = C_::ROWATER * C_::G;
    R AVG_GST = R(1.0) / R(NGST);
    R CONST1 = BETAMAX / ipow(C_::XKAPPA, 2) / C_::ROWATER;
    R NU_AIR = C_::RNUAIR, FAC_NU_AIR = C_::RNUAIRM, FACM1_NU_AIR = R(4.0) / NU_AIR;
    R FU = std::fabs(SWELLF3), FUD = SWELLF2;
    R DELABM1 = R(IAB) / (ABMAX - ABMIN);
    R ABS_TAUWSHELTER = std::fabs(TAUWSHELTER);
    R SIG_N = wsigstar(USTAR, Z0, WSTAR);
    R UORBT = std::numeric_limits<R>::min(), AORB = std::numeric_limits<R>::min();
    std::vector<R> SIG(ml), SIGM1(ml), SIG2(ml), CONST(ml), COEF(ml), COEF5(ml);
    for (int m = 0; m < ml; ++m) {
      SIG[m] = C_::ZPI * fd->FR[m];
      SIGM1[m] = R(1.0) / SIG[m];
      SIG2[m] = ipow(SIG[m], 2);
      R DFIM_SIG2 = fd->DFIM[m] * SIG2[m];
      CONST[m] = SIG[m] * CONST1;
      COEF[m] = -(SWELLF * R(16.) * SIG2[m] / (C_::G * C_::ROWATER));
      COEF5[m] = -(SWELLF5 * R(2.) * std::sqrt(R(2.) * NU_AIR * SIG[m]) / C_::ROWATER);
      R TEMP = F[0 + kl * m];
      for (int k = 1; k < kl; ++k) TEMP = TEMP + F[k + kl * m];
      UORBT = UORBT + DFIM_SIG2 * TEMP;
      AORB = AORB + fd->DFIM[m] * TEMP;
    }
    UORBT = R(2.0) * std::sqrt(UORBT);
    AORB = R(2.0) * std::sqrt(AORB);
    R RE = FACM1_NU_AIR * UORBT * AORB;
    R Z0VIS = FAC_NU_AIR / std::max(USTAR, R(0.0001));
    R Z0TUB = Z0RAT * std::min(Z0TUBMAX, Z0);
    R Z0NOZ = std::max(Z0VIS, Z0TUB);
    R ZORB = AORB / Z0NOZ;
    R XI = (std::log10(std::max(ZORB, R(3.0))) - ABMIN) * DELABM1;
    int IND = std::min(IAB - 1, int_f(XI));
    R DELI1 = std::min(R(1.0), XI - R(IND));
    R DELI2 = R(1.0) - DELI1;
    R FWW = st->SWELLFT[IND - 1] * DELI2 + st->SWELLFT[IND] * DELI1;
    R TEMP2 = FWW * UORBT;
    R RE_C = SWELLF4;                                   // SWELLF6 == 1
    R SMOOTH = R(0.5) * std::tanh((RE - RE_C) / SWELLF7);
    R PTURB = R(0.5) + SMOOTH, PVISC = R(0.5) - SMOOTH;
    R XSTRESS[2] = {0, 0}, YSTRESS[2] = {0, 0}, USG2[2], TAUX[2], TAUY[2];
    USG2[0] = ipow(USTAR * (R(1.0) + SIG_N), 2);
    USG2[1] = ipow(USTAR * (R(1.0) - SIG_N), 2);
    for (int g = 0; g < NGST; ++g) { TAUX[g] = USG2[g] * std::sin(UDIR); TAUY[g] = USG2[g] * std::cos(UDIR); }
    R ROGOROAIR = ROG / std::max(ROAIRN, R(1.0));
    R ROAIRN_PVISC = ROAIRN * PVISC;
    std::vector<R> CM(ml), XK(ml);
    for (int m = 0; m < ml; ++m) {
      if (cfg.shallow_run) { XK[m] = sh->tfak(INDEP, m); CM[m] = XK[m] * SIGM1[m]; }
      else { CM[m] = SIG[m] / C_::G; XK[m] = SIG2[m] / C_::G; }
    }
    const R SHv = R(1.0);
    std::vector<R> COSLP(kl * 2), UFAC(kl * 2), DSTAB(kl * 2);
    for (int m = 0; m < ml; ++m) {
      R USTP[2], USDIRP[2], UCN[2], UCNZALPD[2];
      for (int g = 0; g < NGST; ++g) {
        R TAUPX = TAUX[g] - ABS_TAUWSHELTER * XSTRESS[g];
        R TAUPY = TAUY[g] - ABS_TAUWSHELTER * YSTRESS[g];
        USTP[g] = std::pow(ipow(TAUPX, 2) + ipow(TAUPY, 2), R(0.25));
        USDIRP[g] = std::atan2(TAUPX, TAUPY);
      }
      R CONSTF = ROGOROAIR * CM[m] * fd->DFIM[m];
      for (int g = 0; g < NGST; ++g)
        for (int k = 0; k < kl; ++k) COSLP[k + kl * g] = std::cos(fd->TH[k] - USDIRP[g]);
      for (int g = 0; g < NGST; ++g) { UCN[g] = USTP[g] * CM[m]; UCNZALPD[g] = C_::XKAPPA / (UCN[g] + ZALP); }
      R ZCN = std::log(XK[m] * Z0);
      R CNSN = CONST[m] * SHv * ROAIRN;
      for (int k = 0; k < kl; ++k) LLWS[k + kl * m] = 0;
      for (int g = 0; g < NGST; ++g)
        for (int k = 0; k < kl; ++k) {
          R c = COSLP[k + kl * g];
          if (c > R(0.01)) {
            R X = c * UCN[g];
            R ZLOG = ZCN + UCNZALPD[g] / c;
            if (ZLOG < R(0.0)) {
              R ZLOG2X = ZLOG * ZLOG * X;
              UFAC[k + kl * g] = std::exp(ZLOG) * ZLOG2X * ZLOG2X;
              LLWS[k + kl * m] = 1;
            } else UFAC[k + kl * g] = R(0.0);
          } else UFAC[k + kl * g] = R(0.0);
        }
      R DSTAB1 = COEF5[m] * ROAIRN_PVISC * XK[m];
      R TEMP1 = COEF[m] * ROAIRN;
      for (int g = 0; g < NGST; ++g)
        for (int k = 0; k < kl; ++k) {
          R DSTAB2 = TEMP1 * (TEMP2 + (FU + FUD * COSLP[k + kl * g]) * USTP[g]);
          DSTAB[k + kl * g] = DSTAB1 + PTURB * DSTAB2;
        }
      for (int k = 0; k < kl; ++k) {
        R CONST11 = CONSTF * fd->SINTH[k], CONST22 = CONSTF * fd->COSTH[k];
        R SLP[2], FLP[2];
        for (int g = 0; g < NGST; ++g) { SLP[g] = CNSN * UFAC[k + kl * g]; FLP[g] = SLP[g] + DSTAB[k + kl * g]; }
        for (int g = 0; g < NGST; ++g) {
          SLP[g] = SLP[g] * F[k + kl * m];
          XSTRESS[g] = XSTRESS[g] + SLP[g] * CONST11;
          YSTRESS[g] = YSTRESS[g] + SLP[g] * CONST22;
        }
        R SLP_AVG = SLP[0] + SLP[1], FLP_AVG = FLP[0] + FLP[1];
        SPOS[k + kl * m] = AVG_GST * SLP_AVG;
        FL[k + kl * m] = AVG_GST * FLP_AVG;
        SL[k + kl * m] = FL[k + kl * m] * F[k + kl * m];
      }
    }
  }

  // ---- TAUWINDS :5555-5587 ----------------------------------------------------
  static R tauwinds(const std::vector<R>& S, const std::vector<R>& CINV, const std::vector<R>& DSII) {
    R s = 0;
    for (size_t i = 0; i < S.size(); ++i) s = s + S[i] * CINV[i] * DSII[i];
    return C_::G * C_::ROWATER * s;
  }
  // extension of a direction-integrated spectrum to 10 Hz (LFACTOR :4554-4603,
  // TAU_WAVE_ATMOS :5317-5360); mode 0: plain and positive-part sums, mode 1:
  // |negative part| sums.
  int nk10hz(const std::vector<R>& SIG) const {
    const R FRQMAX = R(10.);
    int n = (int)std::ceil(std::log(FRQMAX / (SIG[0] / C_::ZPI)) / std::log(C_::CO)) + 1;
    return std::max(ML(), n);
  }

  // ---- LFACTOR :4465-4700 ------------------------------------------------------
  // nit (optional): iterations run (0 when the stress needs no reduction);
  // margin: the smallest relative distance of |ERR| from the exit threshold
  // 1.54E-4 over the iterations run (how close the count came to changing).
  void lfactor(const std::vector<R>& S /*[k + KL*m]*/, const std::vector<R>& CINV, R U10, R USTAR, R USDIR, R ROAIRN,
               const std::vector<R>& SIG, const std::vector<R>& DSII, std::vector<R>& LFACT, R& TAUWX, R& TAUWY,
               int* nit = nullptr, double* margin = nullptr) const {
    const int NTH = KL(), NK = ML();
    const R SIN6WS = R(32.); const int ITERMAX = 80;
    int NK10 = nk10hz(SIG);
    std::vector<R> SIG10(NK10), CINV10(NK10), DSII10(NK10), LF10(NK10), SD(NK10), SDX(NK10), SDY(NK10), UCINV10(NK10);
    for (int ik = 0; ik < NK; ++ik) {
      R a = 0, bx = 0, by = 0;
      for (int th = 0; th < NTH; ++th) a = a + S[th + NTH * ik];
      for (int th = 0; th < NTH; ++th) bx = bx + std::max(R(0.), S[th + NTH * ik]) * fd->COSTH[th];
      for (int th = 0; th < NTH; ++th) by = by + std::max(R(0.), S[th + NTH * ik]) * fd->SINTH[th];
      SD[ik] = a * fd->DELTH; SDX[ik] = bx * fd->DELTH; SDY[ik] = by * fd->DELTH;
    }
    if (NK < NK10) {
      for (int i = 0; i < NK10; ++i) SIG10[i] = SIG[0] * std::pow(C_::CO, R(i + 1) - R(1.0));
      for (int i = 0; i < NK; ++i) CINV10[i] = CINV[i];
      for (int i = NK; i < NK10; ++i) CINV10[i] = SIG10[i] * R(0.101978);
      for (int i = 0; i < NK10; ++i) DSII10[i] = R(0.5) * SIG10[i] * (C_::CO - R(1.0) / C_::CO);
      DSII10[0] = R(0.5) * SIG10[0] * (C_::CO - R(1.0));
      DSII10[NK10 - 1] = R(0.5) * SIG10[NK10 - 1] * (C_::CO - R(1.0)) / C_::CO;
      for (int i = NK; i < NK10; ++i) {
        R r = ipow(SIG10[NK - 1] / SIG10[i], 2);
        SD[i] = SD[NK - 1] * r; SDX[i] = SDX[NK - 1] * r; SDY[i] = SDY[NK - 1] * r;
      }
    } else {
      for (int i = 0; i < NK; ++i) { SIG10[i] = SIG[i]; CINV10[i] = CINV[i]; DSII10[i] = DSII[i]; }
    }
    R TAU_TOT = ipow(USTAR, 2) * ROAIRN;
    R TAU_VIS = std::max(R(0.0), -(R(5.0E-5) * U10) + R(1.1E-3)) * ipow(U10, 2) * ROAIRN;
    TAU_VIS = std::min(R(0.95) * TAU_TOT, TAU_VIS);
    R TAUVX = TAU_VIS * crcos(USDIR), TAUVY = TAU_VIS * crsin(USDIR);
    TAUWX = tauwinds(SDX, CINV10, DSII10);
    TAUWY = tauwinds(SDY, CINV10, DSII10);
    R TAUX = TAUVX + TAUWX, TAUY = TAUVY + TAUWY;
    R TAU = std::sqrt(ipow(TAUX, 2) + ipow(TAUY, 2));
    R ERR = (TAU - TAU_TOT) / TAU_TOT;
    for (auto& v : LF10) v = R(1.0);
    int NIT = 0;
    double MARGIN = 1e30;
    if (TAU > TAU_TOT) {
      bool OVERSHOT = false;
      R RTAU = ERR / R(90.);
      R DRTAU = R(2.0);
      int SIGN_NEW = (int)fsign(R(1.0), ERR);
      R UPROXY = SIN6WS * USTAR;
      for (int i = 0; i < NK10; ++i) UCINV10[i] = R(1.0) - (UPROXY * CINV10[i]);
      std::vector<R> tx(NK10), ty(NK10);
      for (int it = 1; it <= ITERMAX; ++it) {
        NIT = it;
        for (int i = 0; i < NK10; ++i) LF10[i] = std::min(R(1.0), crexp(UCINV10[i] * RTAU));
        for (int i = 0; i < NK10; ++i) { tx[i] = SDX[i] * LF10[i]; ty[i] = SDY[i] * LF10[i]; }
        TAUWX = tauwinds(tx, CINV10, DSII10);
        TAUWY = tauwinds(ty, CINV10, DSII10);
        TAUX = TAUVX + TAUWX; TAUY = TAUVY + TAUWY;
        TAU = std::sqrt(ipow(TAUX, 2) + ipow(TAUY, 2));
        ERR = (TAU - TAU_TOT) / TAU_TOT;
        int SIGN_OLD = SIGN_NEW;
        SIGN_NEW = (int)fsign(R(1.0), ERR);
        if (SIGN_NEW != SIGN_OLD) OVERSHOT = true;
        if (OVERSHOT) DRTAU = std::max(R(0.5) * (R(1.0) + DRTAU), R(1.00010));
        RTAU = RTAU * ipow(DRTAU, SIGN_NEW);
        MARGIN = std::min(MARGIN, std::fabs(std::fabs((double)ERR) - (double)R(1.54E-4)) / (double)R(1.54E-4));
        if (std::fabs(ERR) < R(1.54E-4)) break;
      }
    }
    if (nit) *nit = NIT;
    if (margin) *margin = MARGIN;
    LFACT.resize(NK);
    for (int i = 0; i < NK; ++i) LFACT[i] = LF10[i];
  }

  // ---- TAU_WAVE_ATMOS :5258-5368 ------------------------------------------------
  void tau_wave_atmos(const std::vector<R>& S, const std::vector<R>& CINV, const std::vector<R>& SIG,
                      const std::vector<R>& DSII, R& TAUNWX, R& TAUNWY) const {
    const int NTH = KL(), NK = ML();
    int NK10 = nk10hz(SIG);
    std::vector<R> SIG10(NK10), CINV10(NK10), DSII10(NK10), SDX(NK10), SDY(NK10);
    for (int ik = 0; ik < NK; ++ik) {
      R bx = 0, by = 0;
      for (int th = 0; th < NTH; ++th) bx = bx + std::fabs(std::min(R(0.), S[th + NTH * ik])) * fd->COSTH[th];
      for (int th = 0; th < NTH; ++th) by = by + std::fabs(std::min(R(0.), S[th + NTH * ik])) * fd->SINTH[th];
      SDX[ik] = bx * fd->DELTH; SDY[ik] = by * fd->DELTH;
    }
    if (NK < NK10) {
      for (int i = 0; i < NK10; ++i) SIG10[i] = SIG[0] * std::pow(C_::CO, R(i + 1) - R(1.0));
      for (int i = 0; i < NK; ++i) CINV10[i] = CINV[i];
      for (int i = NK; i < NK10; ++i) CINV10[i] = SIG10[i] * R(0.101978);
      for (int i = 0; i < NK10; ++i) DSII10[i] = R(0.5) * SIG10[i] * (C_::CO - R(1.0) / C_::CO);
      DSII10[0] = R(0.5) * SIG10[0] * (C_::CO - R(1.0));
      DSII10[NK10 - 1] = R(0.5) * SIG10[NK10 - 1] * (C_::CO - R(1.0)) / C_::CO;
      for (int i = NK; i < NK10; ++i) {
        R r = ipow(SIG10[NK - 1] / SIG10[i], 2);
        SDX[i] = SDX[NK - 1] * r; SDY[i] = SDY[NK - 1] * r;
      }
    } else {
      for (int i = 0; i < NK; ++i) { SIG10[i] = SIG[i]; CINV10[i] = CINV[i]; DSII10[i] = DSII[i]; }
    }
    TAUNWX = tauwinds(SDX, CINV10, DSII10);
    TAUNWY = tauwinds(SDY, CINV10, DSII10);
  }

  // ---- SINPUT_ST6 :4704-4925 --------------------------------------------------
  void sinput_st6(const R* F, const R* CGG, const R* WN, R UABS, R USTAR, R USDIR, R ROAIRN, R& TAUW, R& TAUNW,
                  R* SL, R* SPOS, R* FL, int* nit = nullptr, double* margin = nullptr) const {
    const int NTH = KL(), NK = ML();
    const R SIN6WS = R(32.), SIN6A0 = R(0.09);
    std::vector<R> SIG(NK), DSII(NK);
    for (int m = 0; m < NK; ++m) { SIG[m] = C_::ZPI * fd->FR[m]; DSII[m] = C_::ZPI * fd->DF[m]; }
    R COSU = crcos(USDIR), SINU = crsin(USDIR);
    R TAUNWX = 0, TAUNWY = 0, TAUWX = 0, TAUWY = 0;
    R UPROXY = SIN6WS * USTAR;
    const int NS = NTH * NK;
    std::vector<R> A(NS), Kn(NS), W1(NS), D(NS), S(NS), CINV2(NS), SDENSIG(NS), DINPOS(NS), DINTOT(NS);
    std::vector<R> ADENSIG(NK), KMAX(NK), ANAR(NK), SQRTBN(NK), CINV(NK), LFACT;
    for (int ik = 0; ik < NK; ++ik)
      for (int th = 0; th < NTH; ++th) {
        int i = th + NTH * ik;
        CINV2[i] = WN[ik] / SIG[ik];
        A[i] = F[i] * CGG[ik] / (C_::ZPI * SIG[ik]);
        Kn[i] = A[i];
      }
    for (int ik = 0; ik < NK; ++ik) {
      R s = 0; for (int th = 0; th < NTH; ++th) s = s + Kn[th + NTH * ik];
      ADENSIG[ik] = s * SIG[ik] * fd->DELTH;
      R mx = Kn[NTH * ik]; for (int th = 1; th < NTH; ++th) mx = std::max(mx, Kn[th + NTH * ik]);
      KMAX[ik] = mx;
      for (int th = 0; th < NTH; ++th) {
        if (KMAX[ik] < R(1.0E-34)) Kn[th + NTH * ik] = R(1.);
        else Kn[th + NTH * ik] = Kn[th + NTH * ik] / KMAX[ik];
      }
      R s2 = 0; for (int th = 0; th < NTH; ++th) s2 = s2 + Kn[th + NTH * ik];
      ANAR[ik] = R(1.0) / (s2 * fd->DELTH);
      SQRTBN[ik] = std::sqrt(ANAR[ik] * ADENSIG[ik] * ipow(WN[ik], 3));
    }
    const R RAW = ROAIRN / C_::ROWATER;
    for (int ik = 0; ik < NK; ++ik)
      for (int th = 0; th < NTH; ++th) {
        int i = th + NTH * ik;
        R proj = UPROXY * CINV2[i] * (fd->COSTH[th] * COSU + fd->SINTH[th] * SINU) - R(1.);
        W1[i] = ipow(std::max(R(0.), proj), 2);
        D[i] = RAW * SIG[ik] * (R(2.8) - (R(1.) + std::tanh(R(10.) * SQRTBN[ik] * W1[i] - R(11.)))) * SQRTBN[ik] * W1[i];
        S[i] = D[i] * A[i];
      }
    for (int ik = 0; ik < NK; ++ik) CINV[ik] = CINV2[NTH * ik];
    for (int i = 0; i < NS; ++i) { int ik = i / NTH; SDENSIG[i] = S[i] * SIG[ik] / CGG[ik]; }
    lfactor(SDENSIG, CINV, UABS, USTAR, USDIR, ROAIRN, SIG, DSII, LFACT, TAUWX, TAUWY, nit, margin);
    R sumlf = 0; for (int ik = 0; ik < NK; ++ik) sumlf = sumlf + LFACT[ik];
    if (sumlf < R(NK)) {
      for (int i = 0; i < NS; ++i) D[i] = D[i] * LFACT[i / NTH];
      for (int i = 0; i < NS; ++i) S[i] = D[i] * A[i];
    }
    DINPOS = D;
    {
      for (int ik = 0; ik < NK; ++ik)
        for (int th = 0; th < NTH; ++th) {
          int i = th + NTH * ik;
          R proj = UPROXY * CINV2[i] * (fd->COSTH[th] * COSU + fd->SINTH[th] * SINU) - R(1.);
          R W2 = ipow(std::min(R(0.), proj), 2);
          D[i] = D[i] - (RAW * SIG[ik] * SIN6A0 * (R(2.8) - (R(1.) + std::tanh(R(10.) * SQRTBN[ik] * W2 - R(11.)))) *
                         SQRTBN[ik] * W2);
        }
      DINTOT = D;
      for (int i = 0; i < NS; ++i) S[i] = D[i] * A[i];
      for (int i = 0; i < NS; ++i) { int ik = i / NTH; SDENSIG[i] = S[i] * SIG[ik] / CGG[ik]; }
      tau_wave_atmos(SDENSIG, CINV, SIG, DSII, TAUNWX, TAUNWY);
    }
    TAUW = std::sqrt(ipow(TAUWX, 2) + ipow(TAUWY, 2));
    TAUNW = std::sqrt(ipow(TAUNWX, 2) + ipow(TAUNWY, 2));
    for (int i = 0; i < NS; ++i) { SL[i] = DINTOT[i] * F[i]; SPOS[i] = DINPOS[i] * F[i]; FL[i] = DINTOT[i]; }
  }

  // ---- WAVNU2 :4343-4461 ---------------------------------------------------------
  void wavnu2(R DEPTH, R* WN, R* CGG) const {
    const R EPS = R(1E-7); const int NMAX = 15;
    for (int m = 0; m < ML(); ++m) {
      R SIG = C_::ZPI * fd->FR[m], H = DEPTH;
      R W0 = std::fabs(SIG), Kk, KOLD = 0, CG;
      if (W0 < std::sqrt(C_::G / H)) Kk = W0 / std::sqrt(C_::G * H);
      else Kk = W0 * W0 / C_::G;
      bool conv = false;
      for (int i = 1; i <= NMAX; ++i) {
        R DIF = std::fabs(Kk - KOLD);
        R RDIF = (Kk != R(0)) ? DIF / Kk : R(0);
        if (DIF < EPS && RDIF < EPS) { conv = true; break; }
        KOLD = Kk;
        R F1 = C_::G * KOLD * crtanh(KOLD * H) - ipow(W0, 2);
        R FD;
        if (KOLD * H > R(25)) FD = C_::G * crtanh(KOLD * H);
        else FD = C_::G * crtanh(KOLD * H) + C_::G * KOLD * H / ipow(crcosh(KOLD * H), 2);
        Kk = KOLD - F1 / FD;
      }
      (void)conv;
      if (R(2) * Kk * H > R(25)) CG = W0 / Kk * R(0.5);
      else CG = W0 / Kk * R(0.5) * (R(1) + (R(2) * Kk * H / crsinh(R(2) * Kk * H)));
      if (SIG < R(0.0)) { Kk = -Kk; CG = -CG; }
      WN[m] = Kk; CGG[m] = CG;
    }
  }

  // ---- FRCUTINDEX :3569-3647 and FRCUTINDEX_ST6 :5447-5515 -----------------------
  // arg (optional) receives the REAL value that NINT / INT rounds.
  int frcutindex(R FM, R FMWS, R USTAR, double* arg = nullptr) const {
    const R EPSUS = R(1.0E-6), FRIC = R(28.0), TAILFACTOR = R(2.5), TAILFACTOR_PM = R(3.0);
    R FPMH = TAILFACTOR / fd->FR[0];
    R FPPM = TAILFACTOR_PM * C_::G / (FRIC * C_::ZPI * fd->FR[0]);
    R FM2 = std::max(FMWS, FM) * FPMH;
    R FPM = FPPM / std::max(USTAR, EPSUS);
    R FPM4 = std::max(FM2, FPM);
    R X = crlog10(FPM4) * fd->INV_LOG_CO;
    if (arg) *arg = (double)X;
    int MIJ = nint_f(X) + 1;
    return std::min(std::max(1, MIJ), ML());
  }
  int frcutindex_st6(R FMEAN, R USTAR, double* arg = nullptr) const {
    const int NK = ML();
    const R SIN6FC = R(6.);
    R FXFM = SIN6FC; FXFM = FXFM * C_::ZPI;
    R FXPM = R(4.0); FXPM = FXPM * C_::G / R(28.);
    R SIGNK = C_::ZPI * fd->FR[NK - 1];
    R FHIGH = std::max(FXFM * FMEAN, FXPM / USTAR);
    R FACTI1 = R(1.) / crlog(C_::CO);
    R FACTI2 = R(1.) - crlog(C_::ZPI * fd->FR[0]) * FACTI1;
    int NKH = std::min(NK, int_f(FACTI2 + FACTI1 * crlog(std::max(R(1.E-7), FHIGH))));
    int NKH1 = std::min(NK, NKH + 1);
    FHIGH = std::min(SIGNK, std::max(FXFM * FMEAN, FXPM / USTAR));
    R X = FACTI2 + FACTI1 * crlog(std::max(R(1.E-7), FHIGH));
    if (arg) *arg = (double)X;
    NKH = std::max(2, std::min(NKH1, int_f(X)));
    return NKH;
  }

  // ---- TAU_PHI_HF :3853-3966 (XLEVTAIL = 0 as passed by STRESSO) -----------------
  void tau_phi_hf(int MIJ, R USTAR, R Z0, R& TAUHF, R& PHIHF) const {
    const int JT = SourceTables<R>::JTOT_TAUHF; const R ZSUP = R(0.0), XLEVTAIL = R(0.0);
    R GM1 = R(1.0) / C_::G;
    R X0G = st->X0TAUHF * C_::G;
    R OMEGAC = C_::ZPI * fd->FR[MIJ - 1];
    R UST0 = USTAR, TAUW0 = ipow(UST0, 2);
    R GZ0 = C_::G * Z0, XLOGGZ0 = std::log(GZ0);
    R OMEGACC = std::max(OMEGAC, X0G / UST0);
    R SQRTZ0OG = std::sqrt(Z0 * GM1), SQRTGZ0 = R(1.0) / SQRTZ0OG;
    R YC = OMEGACC * SQRTZ0OG, ZINF = std::log(YC);
    R DELZ = std::max((ZSUP - ZINF) / R(JT - 1), R(0.0));
    TAUHF = R(0.0); PHIHF = R(0.0);
    R TAUW = TAUW0, UST = UST0;
    for (int J = 1; J <= JT; ++J) {
      R Y = std::exp(ZINF + R(J - 1) * DELZ);
      R OMEGA = Y * SQRTGZ0;
      R CM1 = OMEGA * GM1;
      R ZX = UST * CM1 + ZALP;
      R ZARG = C_::XKAPPA / ZX;
      R ZLOG = XLOGGZ0 + R(2.0) * std::log(CM1) + ZARG;
      ZLOG = std::min(ZLOG, R(0.0));
      R ZBETA = std::exp(ZLOG) * ipow(ZLOG, 4);
      R FNC2 = ZBETA * TAUW * st->WTAUHF[J - 1] * DELZ;
      TAUW = std::max(TAUW - XLEVTAIL * FNC2, R(0.0));
      UST = std::sqrt(TAUW);
      TAUHF = TAUHF + FNC2;
      PHIHF = PHIHF + FNC2 / Y;
    }
    PHIHF = SQRTZ0OG * PHIHF;
  }

  // ---- STRESSO :3164-3356 ---------------------------------------------------------
  void stresso(const R* F, const R* SPOS, R USTAR, R UDIR, R Z0, int MIJ, R& TAUW, R& PHIAW, int INDEP) const {
    const int kl = KL(), ml = ML();
    R UST2 = ipow(USTAR, 2);
    R GM1 = R(1.0) / C_::G;
    R CONST = fd->DELTH * ipow(C_::ZPI, 4) * GM1;
    R CONST1 = CONST * fd->FR5[MIJ - 1] * GM1;
    R CONST2 = C_::ROAIR * CONST * fd->FR5[MIJ - 1];
    std::vector<R> CM(ml), RHOWGDFTH(ml);
    for (int m = 0; m < ml; ++m) {
      if (cfg.shallow_run) { R SIGM1 = R(1.0) / (C_::ZPI * fd->FR[m]); CM[m] = sh->tfak(INDEP, m) * SIGM1; }
      else { R SIG = C_::ZPI * fd->FR[m]; CM[m] = SIG * GM1; }
    }
    for (int m = 0; m < MIJ; ++m) RHOWGDFTH[m] = fd->RHOWG_DFIM[m];
    if (MIJ != ml) RHOWGDFTH[MIJ - 1] = R(0.5) * RHOWGDFTH[MIJ - 1];
    for (int m = MIJ; m < ml; ++m) RHOWGDFTH[m] = R(0.0);
    PHIAW = 0; R XSTRESS = 0, YSTRESS = 0;
    for (int m = 0; m < MIJ; ++m) {
      R SINPLUS = std::max(SPOS[0 + kl * m], R(0.));
      R SUMT = SINPLUS, SUMX = SINPLUS * fd->SINTH[0], SUMY = SINPLUS * fd->COSTH[0];
      for (int k = 1; k < kl; ++k) {
        SINPLUS = std::max(SPOS[k + kl * m], R(0.));
        SUMT = SUMT + SINPLUS; SUMX = SUMX + SINPLUS * fd->SINTH[k]; SUMY = SUMY + SINPLUS * fd->COSTH[k];
      }
      PHIAW = PHIAW + SUMT * RHOWGDFTH[m];
      R CMR = CM[m] * RHOWGDFTH[m];
      XSTRESS = XSTRESS + SUMX * CMR;
      YSTRESS = YSTRESS + SUMY * CMR;
    }
    XSTRESS = XSTRESS / std::max(C_::ROAIR, R(1.));
    YSTRESS = YSTRESS / std::max(C_::ROAIR, R(1.));
    R COSW = std::max(std::cos(fd->TH[0] - UDIR), R(0.));
    R TEMP2 = F[0 + kl * (MIJ - 1)] * ipow(COSW, 2);
    R TEMP1 = TEMP2 * COSW;
    for (int k = 1; k < kl; ++k) {
      COSW = std::max(std::cos(fd->TH[k] - UDIR), R(0.));
      TEMP1 = TEMP1 + F[k + kl * (MIJ - 1)] * ipow(COSW, 3);
      TEMP2 = TEMP2 + F[k + kl * (MIJ - 1)] * ipow(COSW, 2);
    }
    R TAU1, PHI1;
    tau_phi_hf(MIJ, USTAR, Z0, TAU1, PHI1);
    R TAUHF = CONST1 * TEMP1 * TAU1;
    R PHIHF = CONST2 * TEMP2 * PHI1;
    PHIAW = PHIAW + PHIHF;
    XSTRESS = XSTRESS + TAUHF * std::sin(UDIR);
    YSTRESS = YSTRESS + TAUHF * std::cos(UDIR);
    TAUW = std::sqrt(ipow(XSTRESS, 2) + ipow(YSTRESS, 2));
    TAUW = std::min(TAUW, UST2 - C_::EPS1);
    TAUW = std::max(TAUW, R(0.));
  }

  // ---- IMPHFTAIL :3651-3731 --------------------------------------------------------
  void imphftail(int MIJ, int INDEP, R* F) const {
    const int kl = KL(), ml = ML();
    std::vector<R> TEMP2(ml);
    for (int m = MIJ - 1; m < ml; ++m) {
      if (cfg.shallow_run) { R AKM1 = R(1.) / sh->tfak(INDEP, m); TEMP2[m] = ipow(AKM1, 3) / sh->tcgond(INDEP, m); }
      else TEMP2[m] = fd->FRM5[m];
    }
    for (int m = MIJ; m < ml; ++m) TEMP2[m] = TEMP2[m] / TEMP2[MIJ - 1];
    for (int k = 0; k < kl; ++k) {
      R TFAC = F[k + kl * (MIJ - 1)];
      for (int m = MIJ; m < ml; ++m) F[k + kl * m] = TEMP2[m] * TFAC;
    }
  }

  // ---- SDISSIP_ARD :1704-1962 (SSDSC3 = SSDSC5 = 0 branches are dead code) -----------
  void sdissip_ard(const R* F, R* SL, R* FL, int INDEP) const {
    const int kl = KL(), ml = ML();
    R TPIINV = R(1.0) / C_::ZPI, TPIINVH = R(0.5) * TPIINV;
    R TMP03 = R(1.0) / (C_::SDSBR * C_::MICHE);
    R SSDSC6M1 = R(1.) - C_::SSDSC6;
    int NW = st->NSDSNTH * 2 + 1;
    std::vector<R> BTH(kl * ml, R(0)), BTH0(ml, R(0)), FACSAT(ml);
    for (int m = 0; m < ml; ++m) {
      R SIG = C_::ZPI * fd->FR[m];
      if (cfg.shallow_run) { R XK = sh->tfak(INDEP, m); FACSAT[m] = ipow(XK, 3) * TPIINV * sh->tcgond(INDEP, m); }
      else { R XK = ipow(SIG, 2) / C_::G; FACSAT[m] = ipow(XK, 3) * TPIINVH * C_::G / SIG; }
    }
    for (int m = 0; m < ml; ++m)
      for (int k = 0; k < kl; ++k) {
        R b = R(0.0);
        for (int k2 = 0; k2 < NW; ++k2) {
          int KK = st->INDICESSAT[k + kl * k2];
          b = b + st->SATWEIGHTS[k + kl * k2] * F[(KK - 1) + kl * m];
        }
        b = b * FACSAT[m];
        BTH[k + kl * m] = b;
        BTH0[m] = std::max(BTH0[m], b);
      }
    for (int m = 0; m < ml; ++m) {
      R SIG = C_::ZPI * fd->FR[m];
      R SSDSC2_SIG = C_::SSDSC2 * SIG;
      R TEMP1 = C_::SSDSC6 * ipow(std::max(R(0.), BTH0[m] * TMP03 - C_::SSDSC4), C_::IPSAT);
      for (int k = 0; k < kl; ++k) {
        R D = SSDSC2_SIG * (TEMP1 + SSDSC6M1 * ipow(std::max(R(0.), BTH[k + kl * m] * TMP03 - C_::SSDSC4), C_::IPSAT));
        SL[k + kl * m] = SL[k + kl * m] + D * F[k + kl * m];
        FL[k + kl * m] = FL[k + kl * m] + D;
      }
    }
  }

  // ---- SDISSIP_ST6 :4929-5102 --------------------------------------------------------
  void sdissip_st6(const R* F, const R* CGG, const R* WN, R* SL, R* FL) const {
    const int NTH = KL(), NK = ML();
    const R SDS6A1 = R(4.75E-6), SDS6A2 = R(7.00E-5);
    const R ANAR = R(1.0), BNT = ipow(R(0.035), 2);
    std::vector<R> T1(NK), T2(NK), ADF(NK), DFII(NK);
    R XFAC = (R(1.0) - R(1.0) / C_::CO) / (C_::CO - R(1.0) / C_::CO);
    for (int ik = 0; ik < NK; ++ik) {
      R ETDENS = (C_::ZPI * BNT) / (ANAR * CGG[ik] * ipow(WN[ik], 3));
      R s = 0; for (int th = 0; th < NTH; ++th) s = s + F[th + NTH * ik];
      R EDENS = s * fd->DELTH;
      R EXDENS = std::max(R(0.0), EDENS - ETDENS);
      R NEXDENS = EXDENS / ETDENS;
      T1[ik] = SDS6A1 * ANAR * fd->FR[ik] * ipow(NEXDENS, 4);
      ADF[ik] = ANAR * ipow(NEXDENS, 4);
    }
    for (int ik = 0; ik < NK; ++ik) {
      DFII[ik] = fd->DF[ik];
      if (ik > 0 && ik < NK - 1) DFII[ik] = DFII[ik] * XFAC;
      R s = 0; for (int j = 0; j <= ik; ++j) s = s + ADF[j] * DFII[j];
      T2[ik] = SDS6A2 * s;
    }
    for (int ik = 0; ik < NK; ++ik) {
      R T12 = R(-1.0) * (std::max(R(0.0), T1[ik]) + std::max(R(0.0), T2[ik]));
      for (int th = 0; th < NTH; ++th) {
        SL[th + NTH * ik] = SL[th + NTH * ik] + T12 * F[th + NTH * ik];
        FL[th + NTH * ik] = FL[th + NTH * ik] + T12;
      }
    }
  }

  // ---- W3SWL6 :5106-5252 -----------------------------------------------------------------
  void w3swl6(const R* F, const R* CGG, const R* WN, R* SL, R* FL) const {
    const int NTH = KL(), NK = ML();
    const R SWL6B1 = R(0.0041);
    std::vector<R> SIG(NK), DDEN(NK), ABAND(NK), BN(NK), DDIS(NK, R(0.)), Kn(NTH * NK);
    for (int m = 0; m < NK; ++m) { SIG[m] = C_::ZPI * fd->FR[m]; DDEN[m] = C_::ZPI * fd->DFIM[m] * SIG[m]; }
    for (int ik = 0; ik < NK; ++ik) {
      R s = 0;
      for (int th = 0; th < NTH; ++th) {
        R a = F[th + NTH * ik] * CGG[ik] / (C_::ZPI * SIG[ik]);
        Kn[th + NTH * ik] = a;
        s = s + a;
      }
      ABAND[ik] = s;
    }
    for (int ik = 0; ik < NK; ++ik) {
      R mx = Kn[NTH * ik]; for (int th = 1; th < NTH; ++th) mx = std::max(mx, Kn[th + NTH * ik]);
      for (int th = 0; th < NTH; ++th) {
        if (mx < R(1.0E-34)) Kn[th + NTH * ik] = R(1.);
        else Kn[th + NTH * ik] = Kn[th + NTH * ik] / mx;
      }
      R s = 0; for (int th = 0; th < NTH; ++th) s = s + Kn[th + NTH * ik];
      R ANAR = R(1.0) / (s * fd->DELTH);
      BN[ik] = ANAR * (ABAND[ik] * SIG[ik] * fd->DELTH) * ipow(WN[ik], 3);
    }
    int IK = 0;
    for (int ik = 1; ik < NK; ++ik) if (ABAND[ik] > ABAND[IK]) IK = ik;
    R s = 0; for (int ik = 0; ik < NK; ++ik) s = s + ABAND[ik] * DDEN[ik] / CGG[ik];
    R B1 = SWL6B1 * (R(2.) * std::sqrt(s) * WN[IK]);
    for (int ik = 0; ik < NK; ++ik)
      if (ABAND[ik] > R(1.E-30)) DDIS[ik] = -(R(2.) / R(3.) * B1 * SIG[ik] * std::sqrt(BN[ik]));
    for (int ik = 0; ik < NK; ++ik)
      for (int th = 0; th < NTH; ++th) {
        SL[th + NTH * ik] = SL[th + NTH * ik] + DDIS[ik] * F[th + NTH * ik];
        FL[th + NTH * ik] = FL[th + NTH * ik] + DDIS[ik];
      }
  }

  // ---- SNONLIN (DIA) :2742-3047 --------------------------------------------------------
  void snonlin(const R* F, R* SL, R* FL, R DEPTH, R AKMEAN, int ij) const {
    const int kl = KL(), ml = ML();
    const DiaTables<R>& T = *dia;
    R ENHFR = R(1);
    if (cfg.shallow_run && cfg.isnonlin == 0) {
      ENHFR = std::max(R(0.75) * DEPTH * AKMEAN, R(.5));
      ENHFR = R(1.) + (R(5.5) / ENHFR) * (R(1.) - R(.833) * ENHFR) * std::exp(R(-1.25) * ENHFR);
    }
    int MFR1STFR = -T.MFRSTLW + 1;
    int MFRLSTFR = ml - T.KFRH + MFR1STFR;
    auto f = [&](int k, int m) { return F[(k - 1) + kl * (m - 1)]; };
    auto sl = [&](int k, int m) -> R& { return SL[(k - 1) + kl * (m - 1)]; };
    auto fl = [&](int k, int m) -> R& { return FL[(k - 1) + kl * (m - 1)]; };
    for (int MC = 1; MC <= T.MLSTHG; ++MC) {
      int MP = T.ikp(MC), MP1 = T.ikp1(MC), MM = T.ikm(MC), MM1 = T.ikm1(MC);
      const int* ic = &T.INLCOEF[5 * (MC - 1)];
      int IC = ic[0], IP = ic[1], IP1 = ic[2], IM = ic[3], IM1 = ic[4];
      const R* rc = &T.RNLCOEF[25 * (MC - 1)];
      R FTAIL = rc[0], GW1 = rc[1], GW2 = rc[2], GW3 = rc[3], GW4 = rc[4];
      R FKLAMPA = rc[5], FKLAMPB = rc[6], FKLAMP2 = rc[7], FKLAMP1 = rc[8];
      R FKLAPA2 = rc[9], FKLAPB2 = rc[10], FKLAP12 = rc[11], FKLAP22 = rc[12];
      R GW5 = rc[13], GW6 = rc[14], GW7 = rc[15], GW8 = rc[16];
      R FKLAMMA = rc[17], FKLAMMB = rc[18], FKLAMM2 = rc[19], FKLAMM1 = rc[20];
      R FKLAMA2 = rc[21], FKLAMB2 = rc[22], FKLAM12 = rc[23], FKLAM22 = rc[24];
      R FTEMP;
      if (cfg.shallow_run) {
        R enh = (cfg.isnonlin == 0) ? ENHFR : ENH_table[(size_t)ij + (size_t)enh_nsea * (MC - 1)];
        FTEMP = T.AF11[MC - T.MFRSTLW] * enh;
      } else FTEMP = T.AF11[MC - T.MFRSTLW];
      int regime = (MC > MFR1STFR && MC < MFRLSTFR) ? 0 : (MC >= MFRLSTFR ? 1 : 2);
      for (int KH = 1; KH <= 2; ++KH)
        for (int k = 1; k <= kl; ++k) {
          int K1 = T.K1W[(k - 1) + kl * (KH - 1)], K2 = T.K2W[(k - 1) + kl * (KH - 1)];
          int K11 = T.K11W[(k - 1) + kl * (KH - 1)], K21 = T.K21W[(k - 1) + kl * (KH - 1)];
          R SAP = GW1 * f(K1, IP) + GW2 * f(K11, IP) + GW3 * f(K1, IP1) + GW4 * f(K11, IP1);
          R SAM = GW5 * f(K2, IM) + GW6 * f(K21, IM) + GW7 * f(K2, IM1) + GW8 * f(K21, IM1);
          R FIJ = (regime == 0) ? f(k, IC) : f(k, IC) * FTAIL;
          R FAD1 = FIJ * (SAP + SAM);
          R FAD2 = FAD1 - R(2.) * SAP * SAM;
          FAD1 = FAD1 + FAD2;
          R FCEN = FTEMP * FIJ;
          R AD = FAD2 * FCEN;
          R DELAD = FAD1 * FTEMP;
          R DELAP = (FIJ - R(2.) * SAM) * T.DAL1 * FCEN;
          R DELAM = (FIJ - R(2.) * SAP) * T.DAL2 * FCEN;
          if (regime == 0) {
            sl(k, MC) = sl(k, MC) - R(2.) * AD;           fl(k, MC) = fl(k, MC) - R(2.) * DELAD;
            sl(K2, MM) = sl(K2, MM) + AD * FKLAMM1;        fl(K2, MM) = fl(K2, MM) + DELAM * FKLAM12;
            sl(K21, MM) = sl(K21, MM) + AD * FKLAMM2;      fl(K21, MM) = fl(K21, MM) + DELAM * FKLAM22;
            sl(K2, MM1) = sl(K2, MM1) + AD * FKLAMMA;      fl(K2, MM1) = fl(K2, MM1) + DELAM * FKLAMA2;
            sl(K21, MM1) = sl(K21, MM1) + AD * FKLAMMB;    fl(K21, MM1) = fl(K21, MM1) + DELAM * FKLAMB2;
            sl(K1, MP) = sl(K1, MP) + AD * FKLAMP1;        fl(K1, MP) = fl(K1, MP) + DELAP * FKLAP12;
            sl(K11, MP) = sl(K11, MP) + AD * FKLAMP2;      fl(K11, MP) = fl(K11, MP) + DELAP * FKLAP22;
            sl(K1, MP1) = sl(K1, MP1) + AD * FKLAMPA;      fl(K1, MP1) = fl(K1, MP1) + DELAP * FKLAPA2;
            sl(K11, MP1) = sl(K11, MP1) + AD * FKLAMPB;    fl(K11, MP1) = fl(K11, MP1) + DELAP * FKLAPB2;
          } else if (regime == 1) {
            sl(K2, MM) = sl(K2, MM) + AD * FKLAMM1;        fl(K2, MM) = fl(K2, MM) + DELAM * FKLAM12;
            sl(K21, MM) = sl(K21, MM) + AD * FKLAMM2;      fl(K21, MM) = fl(K21, MM) + DELAM * FKLAM22;
            if (MM1 <= ml) {
              sl(K2, MM1) = sl(K2, MM1) + AD * FKLAMMA;    fl(K2, MM1) = fl(K2, MM1) + DELAM * FKLAMA2;
              sl(K21, MM1) = sl(K21, MM1) + AD * FKLAMMB;  fl(K21, MM1) = fl(K21, MM1) + DELAM * FKLAMB2;
              if (MC <= ml) {
                sl(k, MC) = sl(k, MC) - R(2.) * AD;        fl(k, MC) = fl(k, MC) - R(2.) * DELAD;
                if (MP <= ml) {
                  sl(K1, MP) = sl(K1, MP) + AD * FKLAMP1;  fl(K1, MP) = fl(K1, MP) + DELAP * FKLAP12;
                  sl(K11, MP) = sl(K11, MP) + AD * FKLAMP2; fl(K11, MP) = fl(K11, MP) + DELAP * FKLAP22;
                  if (MP1 <= ml) {
                    sl(K1, MP1) = sl(K1, MP1) + AD * FKLAMPA;   fl(K1, MP1) = fl(K1, MP1) + DELAP * FKLAPA2;
                    sl(K11, MP1) = sl(K11, MP1) + AD * FKLAMPB; fl(K11, MP1) = fl(K11, MP1) + DELAP * FKLAPB2;
                  }
                }
              }
            }
          } else {
            if (MM1 >= 1) {
              sl(K2, MM1) = sl(K2, MM1) + AD * FKLAMMA;    fl(K2, MM1) = fl(K2, MM1) + DELAM * FKLAMA2;
              sl(K21, MM1) = sl(K21, MM1) + AD * FKLAMMB;  fl(K21, MM1) = fl(K21, MM1) + DELAM * FKLAMB2;
            }
            sl(k, MC) = sl(k, MC) - R(2.) * AD;            fl(k, MC) = fl(k, MC) - R(2.) * DELAD;
            sl(K1, MP) = sl(K1, MP) + AD * FKLAMP1;        fl(K1, MP) = fl(K1, MP) + DELAP * FKLAP12;
            sl(K11, MP) = sl(K11, MP) + AD * FKLAMP2;      fl(K11, MP) = fl(K11, MP) + DELAP * FKLAP22;
            sl(K1, MP1) = sl(K1, MP1) + AD * FKLAMPA;      fl(K1, MP1) = fl(K1, MP1) + DELAP * FKLAPA2;
            sl(K11, MP1) = sl(K11, MP1) + AD * FKLAMPB;    fl(K11, MP1) = fl(K11, MP1) + DELAP * FKLAPB2;
          }
        }
    }
  }

  // ---- MAKE_SHALLOW_SNL :975-1048 ---------------------------------------------------------
  void make_shallow_snl(const R* depth, int nsea) {
    enh_nsea = nsea;
    int MLSTHG = dia->MLSTHG, ml = ML();
    ENH_table.assign((size_t)nsea * MLSTHG, R(0));
    if (cfg.isnonlin == 0) return;
    const R ENH_MAX = R(10.);
    for (int m = 1; m <= ml; ++m)
      for (int ij = 0; ij < nsea; ++ij) {
        R D = depth[ij], OM = C_::ZPI * fd->FR[m - 1], XK = AKI(OM, D);
        ENH_table[ij + (size_t)nsea * (m - 1)] = std::min(ENH_MAX, TRANSF(XK, D));
      }
    for (int m = ml + 1; m <= MLSTHG; ++m)
      for (int ij = 0; ij < nsea; ++ij) {
        R D = depth[ij], OM = C_::ZPI * fd->FR[ml - 1] * ipow(C_::CO, m - ml), XK = AKI(OM, D);
        ENH_table[ij + (size_t)nsea * (m - 1)] = std::min(ENH_MAX, TRANSF(XK, D));
      }
  }

  // ---- SBOTTOM :1527-1589 -------------------------------------------------------------------
  void sbottom(const R* F, R* SL_BOT, R* FL, R DEPTH, int INDEP) const {
    const int kl = KL(), ml = ML();
    const R CONST = R(-2.0) * R(0.038) / C_::G;
    for (int m = 0; m < ml; ++m) {
      R WAV = sh->tfak(INDEP, m);
      R SBO = std::min(R(2.) * DEPTH * WAV, R(50.));
      SBO = CONST * WAV / std::sinh(SBO);
      for (int k = 0; k < kl; ++k) { SL_BOT[k + kl * m] = SL_BOT[k + kl * m] + SBO * F[k + kl * m]; FL[k + kl * m] = FL[k + kl * m] + SBO; }
    }
  }

  // ---- WNFLUXES :3970-4054 ------------------------------------------------------------------
  struct Fluxes { R PHIOC, TAUOC_X, TAUOC_Y, PHIBOT, TAUBOT_X, TAUBOT_Y, PHIAW; };
  void wnfluxes(const R* SL, const R* SL_BOT, R USTAR, R UDIR, R PHIAW, int INDEP, int MIJ, Fluxes& o) const {
    const int kl = KL(), ml = ML();
    R ROG = C_::ROWATER * C_::G;
    o.PHIOC = PHIAW;
    R TAU = C_::ROAIR * ipow(USTAR, 2);
    o.TAUOC_X = TAU * std::sin(UDIR); o.TAUOC_Y = TAU * std::cos(UDIR);
    o.PHIBOT = 0; o.TAUBOT_X = 0; o.TAUBOT_Y = 0;
    std::vector<R> CONSTFM(ml, R(0.));
    R SCDFM = R(0.5) * fd->DELTH * (R(1.) - R(1.) / C_::CO);
    for (int m = 0; m < MIJ - 1; ++m) CONSTFM[m] = ROG * fd->DFIM[m];
    CONSTFM[MIJ - 1] = ROG * SCDFM * fd->FR[MIJ - 1];
    for (int m = 0; m < MIJ; ++m) {
      R CM = cfg.shallow_run ? sh->tfak(INDEP, m) / (C_::ZPI * fd->FR[m]) : C_::ZPI * fd->FR[m] / C_::G;
      for (int k = 0; k < kl; ++k) {
        R s = SL[k + kl * m];
        o.PHIOC = o.PHIOC - s * CONSTFM[m];
        o.TAUOC_X = o.TAUOC_X - CM * s * CONSTFM[m] * fd->SINTH[k];
        o.TAUOC_Y = o.TAUOC_Y - CM * s * CONSTFM[m] * fd->COSTH[k];
        if (cfg.shallow_run) {
          R b = SL_BOT[k + kl * m];
          o.PHIBOT = o.PHIBOT - b * CONSTFM[m];
          o.TAUBOT_X = o.TAUBOT_X - CM * b * CONSTFM[m] * fd->SINTH[k];
          o.TAUBOT_Y = o.TAUBOT_Y - CM * b * CONSTFM[m] * fd->COSTH[k];
        }
      }
    }
  }

  // Integer decisions of one IMPLSCH call and the REAL values they were
  // rounded from: JU (NINT(U10/DELU), :498), the cut-off index MIJ of the
  // first FRCUTINDEX call (:563) and of the last (:697), the LFACTOR
  // iteration count (ST6, :4647-4672; 0 without reduction, -1 for ST4) with
  // the smallest relative distance of |ERR| from its exit threshold, and the
  // wind-sea masks LLWS of the first SINPUT call and of the last one (the
  // mask of the final integrals).
  struct Diag {
    int JU, MIJ1, MIJ2, LFIT;
    double JU_ARG, MIJ1_ARG, MIJ2_ARG, LF_MARGIN;
    uint8_t* LLWS1;  // KL*ML, or null
    uint8_t* LLWS2;
  };

  // ---- IMPLSCH :374-700, one sea point -------------------------------------------------------
  // F: spectrum of the point [k + KL*m], updated in place.
  void implsch_point(R* F, R U10, R UDIR, R& TAUW, R& USTAR, R& Z0, R ROAIRN, R WSTAR, R DEPTH, int INDEP, int ij,
                     Fluxes* flx, Diag* dg = nullptr) const {
    const int kl = KL(), ml = ML(), NS = kl * ml;
    std::vector<R> SL(NS), FL(NS), SPOS(NS), SMIN, SL_BOT, SPRD(kl), WN(ml), CGG(ml);
    std::vector<uint8_t> LLWS(NS);
    for (int k = 0; k < kl; ++k) SPRD[k] = ipow(std::max(R(0.), std::cos(fd->TH[k] - UDIR)), 2);
    const R JU_ARG = U10 / me->DELU;
    int JU = std::min(C_::JUMAX, std::max(nint_f(JU_ARG), 1));
    R EMEAN = total_energy(F, nullptr);
    R FMEAN = femean(F, EMEAN, nullptr);
    R AKMEAN = wm1(F, EMEAN, INDEP);
    if (cfg.iphys == 2) wavnu2(DEPTH, WN.data(), CGG.data());
    R CD, TAUNW = 0, TAUW_DUMMY, PHIAW;
    if (cfg.iphys == 2) w3flx4(U10, USTAR, Z0, CD);
    else airsea(U10, TAUW, USTAR, Z0);
    int LFIT = -1; double LF_MARGIN = 1e30, MIJ_ARG = 0;
    if (cfg.iphys == 1) sinput_ard(F, SL.data(), SPOS.data(), FL.data(), USTAR, UDIR, Z0, ROAIRN, WSTAR, INDEP, LLWS.data());
    else {
      sinput_st6(F, CGG.data(), WN.data(), U10, USTAR, UDIR, ROAIRN, TAUW, TAUNW, SL.data(), SPOS.data(), FL.data(),
                 &LFIT, &LF_MARGIN);
      for (int i = 0; i < NS; ++i) LLWS[i] = SPOS[i] > R(0);
    }
    if (dg && dg->LLWS1) std::copy(LLWS.begin(), LLWS.end(), dg->LLWS1);
    R EMEANWS = total_energy(F, LLWS.data());
    R FMEANWS = femean(F, EMEANWS, LLWS.data());
    int MIJ = (cfg.iphys == 2) ? frcutindex_st6(FMEAN, USTAR, &MIJ_ARG) : frcutindex(FMEAN, FMEANWS, USTAR, &MIJ_ARG);
    if (dg) { dg->JU = JU; dg->JU_ARG = (double)JU_ARG; dg->MIJ1 = MIJ; dg->MIJ1_ARG = MIJ_ARG; dg->LFIT = LFIT; dg->LF_MARGIN = LF_MARGIN; }
    if (cfg.iphys == 2) { stresso(F, SPOS.data(), USTAR, UDIR, Z0, MIJ, TAUW_DUMMY, PHIAW, INDEP); w3flx4(U10, USTAR, Z0, CD); }
    else { stresso(F, SPOS.data(), USTAR, UDIR, Z0, MIJ, TAUW, PHIAW, INDEP); airsea(U10, TAUW, USTAR, Z0); }
    imphftail(MIJ, INDEP, F);
    if (cfg.iphys == 1) sinput_ard(F, SL.data(), SPOS.data(), FL.data(), USTAR, UDIR, Z0, ROAIRN, WSTAR, INDEP, LLWS.data());
    if (cfg.lcflx) { SMIN.resize(NS); for (int i = 0; i < NS; ++i) SMIN[i] = SL[i] - SPOS[i]; }
    if (cfg.iphys == 2) stresso(F, SPOS.data(), USTAR, UDIR, Z0, MIJ, TAUW_DUMMY, PHIAW, INDEP);
    else stresso(F, SPOS.data(), USTAR, UDIR, Z0, MIJ, TAUW, PHIAW, INDEP);
    if (cfg.iphys == 1) sdissip_ard(F, SL.data(), FL.data(), INDEP);
    else { sdissip_st6(F, CGG.data(), WN.data(), SL.data(), FL.data()); w3swl6(F, CGG.data(), WN.data(), SL.data(), FL.data()); }
    snonlin(F, SL.data(), FL.data(), DEPTH, AKMEAN, ij);
    if (cfg.shallow_run) { SL_BOT.assign(NS, R(0.)); sbottom(F, SL_BOT.data(), FL.data(), DEPTH, INDEP); }
    if (cfg.lcflx) {
      std::vector<R> SSOURCE(NS);
      for (int i = 0; i < NS; ++i) SSOURCE[i] = SL[i] - SMIN[i];
      Fluxes o;
      wnfluxes(SSOURCE.data(), cfg.shallow_run ? SL_BOT.data() : nullptr, USTAR, UDIR, PHIAW, INDEP, MIJ, o);
      o.PHIAW = PHIAW;
      if (flx) *flx = o;
    }
    if (cfg.shallow_run) for (int i = 0; i < NS; ++i) SL[i] = SL[i] + SL_BOT[i];
    // implicit update with growth limiter :660-670
    R DELT = R(cfg.idelt);
    for (int m = 0; m < ml; ++m) {
      R DELFL = R(5.0E-07) * C_::G / ipow(fd->FR[m], 4) * DELT;
      R TEMP2 = USTAR * DELFL * std::max(FMEANWS, FMEAN);
      R flmin = me->FLMINFR[(JU - 1) + (size_t)C_::JUMAX * m];
      for (int k = 0; k < kl; ++k) {
        int i = k + kl * m;
        R TEMP1 = DELT * SL[i] / std::max(R(1.), R(1.) - DELT * FL[i]);
        R TEMP3 = std::min(std::fabs(TEMP1), TEMP2);
        F[i] = F[i] + fsign(TEMP3, TEMP1);
        F[i] = std::max(F[i], flmin * SPRD[k]);
      }
    }
    EMEAN = total_energy(F, nullptr);
    FMEAN = femean(F, EMEAN, nullptr);
    EMEANWS = total_energy(F, LLWS.data());
    FMEANWS = femean(F, EMEANWS, LLWS.data());
    MIJ = (cfg.iphys == 2) ? frcutindex_st6(FMEAN, USTAR, &MIJ_ARG) : frcutindex(FMEAN, FMEANWS, USTAR, &MIJ_ARG);
    if (dg) {
      dg->MIJ2 = MIJ; dg->MIJ2_ARG = MIJ_ARG;
      if (dg->LLWS2) std::copy(LLWS.begin(), LLWS.end(), dg->LLWS2);
    }
    imphftail(MIJ, INDEP, F);
  }
};

}  // namespace wamo
