// ORACLE — test infrastructure only (see oracle_tables.hpp header).
//
// Restatement of the integrated output parameters of one sea point:
// COMPUTE_OUTPUT_PARAMETER (wam_output_module.f90:481-640) with the
// interface routines it calls, TOTAL_ENERGY_B (wam_interface_module.f90:
// 1342-1410), FEMEAN (:207-286), TM1_TM2_PERIODS_B (:1152-1245),
// PEAK_PERIOD_B (:741-813), MEAN_DIRECTION_B (:412-533), MEANSQS (:639-737)
// and CHARNOCK_PAR (:159-203); SWELL_SEPARATION (wam_swell_module.f90:
// 106-350) for the wind-sea and swell parameters 17-23 and 25-31 (not its
// partitioning, parameters 41-49).  Kurtosis, radiation stress and Stokes
// drift are not restated.
#pragma once
#include "oracle_tables.hpp"

namespace wamo {

// Parameter numbers of the reference's output BLOCK(:, IP) (CFLAG_P index).
enum OutParam {
  OP_U10 = 1, OP_UDIR = 2, OP_USTAR = 3, OP_CD = 4, OP_CHARNOCK = 5, OP_DEPTH = 6, OP_CUR_SPEED = 7, OP_CUR_DIR = 8,
  OP_HS = 9, OP_TP = 10, OP_TM = 11, OP_TM1 = 12, OP_TM2 = 13, OP_THQ = 14, OP_SPREAD = 15, OP_TAUW_NORM = 16,
  OP_Z0 = 32, OP_MSS = 40,
  // SWELL_SEPARATION: wind sea 17-23, swell 25-31 (Hs, Tp, Tm, TM1, TM2, direction, spread)
  OP_WS_HS = 17, OP_SW_HS = 25
};
constexpr int OUT_NPARAM = 40;  // parameters 1..40 (unset ones stay 0)

template <typename R> struct OutputModel {
  using C_ = K<R>;
  const FreDir<R>* fd; const ShallowTables<R>* sh;
  bool shallow = false;
  bool from = true;  // orientation_of_directions: directions the waves come from (user default, user:537)

  // DEG*x, or MOD(DEG*x + 180, 360) for the "going to" convention
  R orient(R deg) const { return from ? deg : std::fmod(deg + R(180.), R(360.)); }

  // The integrals of one spectrum F[k + KL*m] that COMPUTE_OUTPUT_PARAMETER
  // and SWELL_SEPARATION take: TOTAL_ENERGY (EMEAN), FEMEAN (1/FM), TM1,
  // TM2, PEAK_PERIOD, MEAN_DIRECTION (THQ and SPREAD in degrees).
  struct Integrals { R E, TM, TM1, TM2, TP, THQ, SPREAD; };
  Integrals integrals(const R* F) const {
    const int kl = fd->KL, ml = fd->ML;
    const R DEG = R(180.) / C_::PI;
    Integrals o;
    std::vector<R> TEMP(ml);
    for (int m = 0; m < ml; ++m) { R s = 0; for (int k = 0; k < kl; ++k) s = s + F[k + kl * m]; TEMP[m] = s; }
    R EMEAN = fd->MO_TAIL * TEMP[ml - 1];
    for (int m = 0; m < ml; ++m) EMEAN = EMEAN + TEMP[m] * fd->DFIM[m];
    EMEAN = std::max(EMEAN, C_::EMIN);
    R FM = fd->MM1_TAIL * TEMP[ml - 1];
    for (int m = 0; m < ml; ++m) FM = FM + TEMP[m] * fd->DFIMOFR[m];
    FM = EMEAN / std::max(FM, C_::EMIN);
    o.E = EMEAN;
    o.TM = R(1.) / FM;
    R TM1 = fd->MP1_TAIL * TEMP[ml - 1];
    for (int m = 0; m < ml; ++m) TM1 = TM1 + TEMP[m] * fd->DFIM_FR[m];
    o.TM1 = (EMEAN > C_::EMIN) ? EMEAN / TM1 : R(1.);
    R TM2 = fd->MP2_TAIL * TEMP[ml - 1];
    for (int m = 0; m < ml; ++m) TM2 = TM2 + TEMP[m] * fd->DFIM_FR2[m];
    o.TM2 = (EMEAN > C_::EMIN) ? std::sqrt(EMEAN / TM2) : R(1.);
    int IPEAK = 0;
    for (int m = 1; m < ml; ++m) if (TEMP[m] > TEMP[IPEAK]) IPEAK = m;
    o.TP = (IPEAK == 0) ? R(1.) : R(1.) / fd->FR[IPEAK];
    R SI = 0, CI = 0, SPREAD = 0;
    for (int k = 0; k < kl; ++k) {
      R T = F[k] * fd->DFIM[0];
      for (int m = 1; m < ml; ++m) T = T + F[k + kl * m] * fd->DFIM[m];
      SI = SI + fd->SINTH[k] * T;
      CI = CI + fd->COSTH[k] * T;
      SPREAD = SPREAD + T;
    }
    {
      R ci = (CI == R(0.)) ? R(0.1E-30) : CI;
      R THQ = std::atan2(SI, ci);
      if (THQ < R(0.)) THQ = THQ + C_::ZPI;
      if (THQ > C_::ZPI - R(0.001)) THQ = R(0.);
      o.THQ = orient(THQ * DEG);
    }
    {
      const R lim = R(0.1E-15);
      R ci = (std::fabs(CI) < lim) ? fsign(lim, CI) : CI;
      R si = (std::fabs(SI) < lim) ? fsign(lim, SI) : SI;
      R sp = (std::fabs(SPREAD) < lim) ? fsign(lim, SPREAD) : SPREAD;
      sp = R(2.) * (R(1.) - std::sqrt(ipow(si, 2) + ipow(ci, 2)) / sp);
      sp = (sp <= R(0)) ? std::numeric_limits<R>::min() : std::sqrt(sp);
      o.SPREAD = sp * DEG;
    }
    return o;
  }

  // SWELL_SEPARATION (wam_swell_module.f90:106-350) without the partitioning:
  // a bin is swell where 28/C(M) * 1.2*USTAR*COS(TH(K)-UDIR) < 1 (FL1 =
  // MAX(F, EPSMIN) there, 0 elsewhere), wind sea FL3 - FL1; out[p - 1] for
  // p = 17..23 (wind sea) and 25..31 (swell), the energies as 4*SQRT(E).
  // The cosine is the correctly rounded single-precision value, as the
  // device kernel forms it, so both classify every bin alike.
  void swell(const R* F, R UDIR, R USTAR, R* out) const {
    const int kl = fd->KL, ml = fd->ML;
    const R FRIC = R(28.), EPSMIN = R(0.1E-32);
    std::vector<R> FL1((size_t)kl * ml), FL14((size_t)kl * ml);
    for (int k = 0; k < kl; ++k) {
      const R FLPP = R(1.2) * USTAR * crcos(fd->TH[k] - UDIR);
      for (int m = 0; m < ml; ++m) {
        const R CM = FRIC / fd->C[m];
        const int b = k + kl * m;
        FL1[b] = (CM * FLPP < R(1.0)) ? std::max(F[b], EPSMIN) : R(0.);
      }
    }
    for (size_t b = 0; b < FL1.size(); ++b) FL14[b] = F[b] - FL1[b];
    const Integrals sw = integrals(FL1.data()), ws = integrals(FL14.data());
    auto put = [&](int p0, const Integrals& q) {
      out[p0 - 1] = R(4.) * std::sqrt(q.E);
      out[p0] = q.TP; out[p0 + 1] = q.TM; out[p0 + 2] = q.TM1; out[p0 + 3] = q.TM2;
      out[p0 + 4] = q.THQ; out[p0 + 5] = q.SPREAD;
    };
    put(OP_WS_HS, ws);
    put(OP_SW_HS, sw);
  }

  // out[p - 1] for p = 1..OUT_NPARAM; F[k + KL*m] of one point.
  void point(const R* F, R U10, R UDIR, R USTAR, R TAUW, R Z0, R DEPTH, R U, R V, int INDEP, R* out) const {
    const int kl = fd->KL, ml = fd->ML;
    const R DEG = R(180.) / C_::PI;
    for (int p = 0; p < OUT_NPARAM; ++p) out[p] = R(0.);
    std::vector<R> TEMP(ml);
    for (int m = 0; m < ml; ++m) { R s = 0; for (int k = 0; k < kl; ++k) s = s + F[k + kl * m]; TEMP[m] = s; }
    out[OP_U10 - 1] = U10;
    out[OP_UDIR - 1] = orient(DEG * UDIR);
    out[OP_USTAR - 1] = USTAR;
    R TAU = ipow(USTAR, 2) + R(0.0001);
    out[OP_CD - 1] = TAU / (ipow(U10, 2) + R(0.01));
    out[OP_TAUW_NORM - 1] = TAUW / (TAU * C_::ROAIR);
    out[OP_CHARNOCK - 1] = C_::G * Z0 / std::max(ipow(USTAR, 2), R(1.0E-6));
    out[OP_DEPTH - 1] = shallow ? DEPTH : R(999.);
    out[OP_CUR_SPEED - 1] = std::sqrt(ipow(U, 2) + ipow(V, 2));
    R cd = orient(std::atan2(U, V) * DEG);
    if (cd < R(0.)) cd = cd + R(360.);
    out[OP_CUR_DIR - 1] = cd;
    // TOTAL_ENERGY
    R EMEAN = fd->MO_TAIL * TEMP[ml - 1];
    for (int m = 0; m < ml; ++m) EMEAN = EMEAN + TEMP[m] * fd->DFIM[m];
    EMEAN = std::max(EMEAN, C_::EMIN);
    // FEMEAN
    R FM = fd->MM1_TAIL * TEMP[ml - 1];
    for (int m = 0; m < ml; ++m) FM = FM + TEMP[m] * fd->DFIMOFR[m];
    FM = EMEAN / std::max(FM, C_::EMIN);
    // MEANSQS: CONST1 = 0.*LOG(FC/FS) makes the tail term 0, so SM starts at EPSMIN
    {
      const R XLAMBDAC = R(0.0628), SURFT = R(0.000075), EPSMIN = R(0.1E-32);
      R FS = fd->FR[ml - 1], XKC = C_::ZPI / XLAMBDAC;
      R FC = std::sqrt(C_::G * XKC + SURFT * ipow(XKC, 3)) / C_::ZPI;
      R CONST1 = R(0.) * std::log(FC / FS);
      R CONST2 = CONST1 * ipow(C_::ZPI, 4) * ipow(FS, 5) / ipow(C_::G, 2) * fd->DELTH;
      R SM = std::max(CONST2 * TEMP[ml - 1], EPSMIN);
      if (shallow) {
        for (int m = 0; m < ml; ++m) SM = SM + fd->DFIM[m] * ipow(sh->tfak(INDEP, m), 2) * TEMP[m];
      } else {
        for (int m = 0; m < ml; ++m) {
          R FD = fd->DFIM[m] * ipow(C_::ZPI * fd->FR[m], 4) / ipow(C_::G, 2);
          SM = SM + FD * TEMP[m];
        }
      }
      out[OP_MSS - 1] = SM;
    }
    out[OP_TM - 1] = R(1.) / FM;
    // TM1_TM2_PERIODS
    R TM1 = fd->MP1_TAIL * TEMP[ml - 1];
    for (int m = 0; m < ml; ++m) TM1 = TM1 + TEMP[m] * fd->DFIM_FR[m];
    TM1 = (EMEAN > C_::EMIN) ? EMEAN / TM1 : R(1.);
    R TM2 = fd->MP2_TAIL * TEMP[ml - 1];
    for (int m = 0; m < ml; ++m) TM2 = TM2 + TEMP[m] * fd->DFIM_FR2[m];
    TM2 = (EMEAN > C_::EMIN) ? std::sqrt(EMEAN / TM2) : R(1.);
    out[OP_TM1 - 1] = TM1;
    out[OP_TM2 - 1] = TM2;
    out[OP_HS - 1] = R(4.) * std::sqrt(EMEAN);
    // PEAK_PERIOD: first maximum of the frequency spectrum
    int IPEAK = 0;
    for (int m = 1; m < ml; ++m) if (TEMP[m] > TEMP[IPEAK]) IPEAK = m;
    out[OP_TP - 1] = (IPEAK == 0) ? R(1.) : R(1.) / fd->FR[IPEAK];
    // MEAN_DIRECTION (THQ and SPREAD)
    R SI = 0, CI = 0, SPREAD = 0;
    for (int k = 0; k < kl; ++k) {
      R T = F[k] * fd->DFIM[0];
      for (int m = 1; m < ml; ++m) T = T + F[k + kl * m] * fd->DFIM[m];
      SI = SI + fd->SINTH[k] * T;
      CI = CI + fd->COSTH[k] * T;
      SPREAD = SPREAD + T;
    }
    {
      R ci = (CI == R(0.)) ? R(0.1E-30) : CI;
      R THQ = std::atan2(SI, ci);
      if (THQ < R(0.)) THQ = THQ + C_::ZPI;
      if (THQ > C_::ZPI - R(0.001)) THQ = R(0.);
      out[OP_THQ - 1] = orient(THQ * DEG);
    }
    {
      const R lim = R(0.1E-15);
      R ci = (std::fabs(CI) < lim) ? fsign(lim, CI) : CI;
      R si = (std::fabs(SI) < lim) ? fsign(lim, SI) : SI;
      R sp = (std::fabs(SPREAD) < lim) ? fsign(lim, SPREAD) : SPREAD;
      sp = R(2.) * (R(1.) - std::sqrt(ipow(si, 2) + ipow(ci, 2)) / sp);
      sp = (sp <= R(0)) ? std::numeric_limits<R>::min() : std::sqrt(sp);
      out[OP_SPREAD - 1] = sp * DEG;
    }
    out[OP_Z0 - 1] = Z0;
  }
};

}  // namespace wamo
