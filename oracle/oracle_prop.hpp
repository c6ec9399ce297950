// ORACLE — test infrastructure only (see oracle_tables.hpp header).
//
// Restatement of the propagation path of wam_propagation_module.f90:
//   GRADIENT :182-275, PREPARE_PROPAGATION :279-598, PROPAGS :635-829,
//   PREPARE_PROPAGATION_COEF with its ten PREP_* variants :837-1913,
//   CHECK_CFL :1917-2138.
// Single rank: NINF = NIJS = 1, NSUP = NIJL = NSEA, land slot NINF-1 = 0.
// Point-indexed arrays carry that land slot at index 0 (1-based points).
// L_OBSTRUCTION and dry points (PUT_DRY) are not restated.
#pragma once
#include <atomic>
#include <thread>
#include "oracle_tables.hpp"

namespace wamo {

template <typename R> struct PropModel {
  using C_ = K<R>;
  OracleConfig cfg;
  const FreDir<R>* fd; const ShallowTables<R>* sh;
  int NSEA = 0, KL = 0, ML = 0;
  // grid
  std::vector<int> KLAT, KLON, KFROMIJ;  // KLAT[(ij-1) + NSEA*((ic-1)+2*(j-1))], values 0 = land
  std::vector<R> WLAT, SINPH, COSPH, DELLAM;
  R DELPHI;
  std::vector<R> DCO, DPSN;  // DCO[0..NSEA] (0 = land slot), DPSN[(ij-1) + NSEA*(ic-1)]
  std::vector<R> DEPTH, U, V;  // [0..NSEA], land slot index 0
  std::vector<int> INDEP;      // [0..NSEA]
  std::vector<R> CGOND;        // [ij + (NSEA+1)*m], ij in 0..NSEA
  // coefficients
  bool has_theta = false, has_sigd = false;
  int nic = 1, nj = 1, nlon = 1;
  std::vector<R> COEF_LAT, COEF_LON, COEF_THETA, COEF_SIGD, COEF_SUM;
  int COUNTER = 1; R total_cfl = 0; R cfl_min = 0;

  size_t b(int ij, int k, int m) const { return (size_t)(ij - 1) + (size_t)NSEA * (k - 1 + (size_t)KL * (m - 1)); }
  size_t nb() const { return (size_t)NSEA * KL * ML; }
  R& lat(int ij, int k, int m, int ic, int j) { return COEF_LAT[b(ij, k, m) + nb() * ((ic - 1) + nic * (j - 1))]; }
  R& lon(int ij, int k, int m, int i) { return COEF_LON[b(ij, k, m) + nb() * (i - 1)]; }
  R& theta(int ij, int k, int m, int i) { return COEF_THETA[b(ij, k, m) + nb() * (i - 1)]; }
  R& sigd(int ij, int k, int m, int i) { return COEF_SIGD[b(ij, k, m) + nb() * (i - 1)]; }
  R& csum(int ij, int k, int m) { return COEF_SUM[b(ij, k, m)]; }
  int klat(int ij, int ic, int j) const { return KLAT[(ij - 1) + NSEA * ((ic - 1) + 2 * (j - 1))]; }
  int klon(int ij, int i) const { return KLON[(ij - 1) + NSEA * (i - 1)]; }
  R wlat(int ij, int ic) const { return WLAT[(ij - 1) + NSEA * (ic - 1)]; }
  R dpsn(int ij, int ic) const { return DPSN[(ij - 1) + NSEA * (ic - 1)]; }
  R cgond(int ij, int m) const { return CGOND[ij + (size_t)(NSEA + 1) * (m - 1)]; }
  int kpm(int k, int d) const { return fd->KPM[(k - 1) * 3 + d + 1]; }
  int mpm(int m, int d) const { return fd->MPM[(m - 1) * 3 + d + 1]; }
  int jxo(int k, int i) const { return fd->JXO[(k - 1) * 2 + i - 1]; }
  int jyo(int k, int i) const { return fd->JYO[(k - 1) * 2 + i - 1]; }

  void set_grid(int nsea, const int* klat_, const int* klon_, const R* wlat_, const int* kfromij, int ny,
                const R* sinph, const R* cosph, const R* dellam, R delphi) {
    NSEA = nsea; KL = fd->KL; ML = fd->ML;
    KLAT.assign(klat_, klat_ + (size_t)nsea * 4); KLON.assign(klon_, klon_ + (size_t)nsea * 2);
    WLAT.assign(wlat_, wlat_ + (size_t)nsea * 2); KFROMIJ.assign(kfromij, kfromij + nsea);
    SINPH.assign(sinph, sinph + ny); COSPH.assign(cosph, cosph + ny); DELLAM.assign(dellam, dellam + ny);
    DELPHI = delphi;
    // wam_initial_module.f90:204-214
    DCO.assign(NSEA + 1, R(0)); DPSN.assign((size_t)NSEA * 2, R(1.));
    if (cfg.spherical_run) {
      for (int ij = 1; ij <= NSEA; ++ij) DCO[ij] = R(1.) / COSPH[KFROMIJ[ij - 1] - 1];
      for (int ij = 1; ij <= NSEA; ++ij)
        for (int ic = 1; ic <= 2; ++ic)
          if (klat(ij, ic, 1) != 0) DPSN[(ij - 1) + NSEA * (ic - 1)] = DCO[ij] / DCO[klat(ij, ic, 1)];
    }
    DEPTH.assign(NSEA + 1, R(999.0)); U.assign(NSEA + 1, R(0)); V.assign(NSEA + 1, R(0));
  }
  void set_depth(const R* d) { for (int ij = 1; ij <= NSEA; ++ij) DEPTH[ij] = d[ij - 1]; }
  void set_current(const R* u, const R* v) { for (int ij = 1; ij <= NSEA; ++ij) { U[ij] = u[ij - 1]; V[ij] = v[ij - 1]; } }

  // GRADIENT :182-275 (no dry points)
  void gradient(const std::vector<R>& FIELD, std::vector<R>& D_LAT, std::vector<R>& D_LON) const {
    D_LAT.assign(NSEA + 1, 0); D_LON.assign(NSEA + 1, 0);
    for (int ij = 1; ij <= NSEA; ++ij) {
      int IP = klat(ij, 2, 1), IM = klat(ij, 1, 1);
      if (cfg.reduced_grid) {
        int IP2 = klat(ij, 2, 2), IM2 = klat(ij, 1, 2);
        if (IP != 0 && IM != 0 && IP2 != 0 && IM2 != 0)
          D_LAT[ij] = (wlat(ij, 2) * FIELD[IP] + (R(1.) - wlat(ij, 2)) * FIELD[IP2] - wlat(ij, 1) * FIELD[IM] -
                       (R(1.) - wlat(ij, 1)) * FIELD[IM2]) / (R(2.) * DELPHI);
        else if (IP != 0 && IM != 0) D_LAT[ij] = (FIELD[IP] - FIELD[IM]) / (R(2.) * DELPHI);
        else if (IP2 != 0 && IM2 != 0) D_LAT[ij] = (FIELD[IP2] - FIELD[IM2]) / (R(2.) * DELPHI);
        else D_LAT[ij] = R(0.0);
      } else {
        if (IP != 0 && IM != 0) D_LAT[ij] = (FIELD[IP] - FIELD[IM]) / (R(2.) * DELPHI);
        else D_LAT[ij] = R(0.0);
      }
    }
    for (int ij = 1; ij <= NSEA; ++ij) {
      int IP = klon(ij, 2), IM = klon(ij, 1), KX = KFROMIJ[ij - 1];
      if (IP != 0 && IM != 0) D_LON[ij] = (FIELD[IP] - FIELD[IM]) / (R(2.) * DELLAM[KX - 1]);
      else D_LON[ij] = R(0.0);
    }
  }

  // PREPARE_PROPAGATION :279-598. Returns 0, or -1 when CHECK_CFL finds a negative coefficient.
  int prepare() {
    const int NDEPTH = sh->NDEPTH;
    INDEP.assign(NSEA + 1, 1);
    if (cfg.shallow_run) {
      for (int ij = 1; ij <= NSEA; ++ij) {
        int v = nint_f(std::log(DEPTH[ij] / sh->DEPTHA) / std::log(sh->DEPTHD) + R(1.));
        v = std::max(v, 1); v = std::min(v, NDEPTH);
        INDEP[ij] = v;
      }
      CGOND.assign((size_t)(NSEA + 1) * ML, 0);
      for (int m = 1; m <= ML; ++m) {
        CGOND[0 + (size_t)(NSEA + 1) * (m - 1)] = sh->tcgond(NDEPTH, m - 1);
        for (int ij = 1; ij <= NSEA; ++ij) CGOND[ij + (size_t)(NSEA + 1) * (m - 1)] = sh->tcgond(INDEP[ij], m - 1);
      }
    }
    std::vector<R> THDD, SIDC;  // [(ij-1) + NSEA*((k-1) + KL*(m-1))]
    if (cfg.refraction_d_run || cfg.refraction_c_run) {
      std::vector<R> DDPHI, DDLAM, DUPHI, DULAM, DVPHI, DVLAM;
      if (cfg.shallow_run) {
        gradient(DEPTH, DDPHI, DDLAM);
        if (cfg.spherical_run) for (int ij = 1; ij <= NSEA; ++ij) DDLAM[ij] = DDLAM[ij] * DCO[ij];
      }
      if (cfg.refraction_c_run) {
        gradient(U, DUPHI, DULAM); gradient(V, DVPHI, DVLAM);
        if (cfg.spherical_run)
          for (int ij = 1; ij <= NSEA; ++ij) { DULAM[ij] = DULAM[ij] * DCO[ij]; DVLAM[ij] = DVLAM[ij] * DCO[ij]; }
      }
      std::vector<int> INDEP_G(NSEA + 1, 1);
      if (cfg.shallow_run) {
        for (int ij = 1; ij <= NSEA; ++ij) {
          R D_MEAN = R(4.) * DEPTH[ij]; int IZ = 4;
          int IP = klat(ij, 2, 1), IM = klat(ij, 1, 1);
          if (cfg.reduced_grid) {
            int IP2 = klat(ij, 2, 2), IM2 = klat(ij, 1, 2);
            if (IP != 0 && IM != 0 && IP2 != 0 && IM2 != 0) {
              D_MEAN = D_MEAN + wlat(ij, 2) * DEPTH[IP] + (R(1.) - wlat(ij, 2)) * DEPTH[IP2] + wlat(ij, 1) * DEPTH[IM] +
                       (R(1.) - wlat(ij, 1)) * DEPTH[IM2];
              IZ += 2;
            } else if (IP != 0 && IM != 0) { D_MEAN = D_MEAN + DEPTH[IP] + DEPTH[IM]; IZ += 2; }
            else if (IP2 != 0 && IM2 != 0) { D_MEAN = D_MEAN + DEPTH[IP2] + DEPTH[IM2]; IZ += 2; }
          } else {
            if (IP != 0 && IM != 0) { D_MEAN = D_MEAN + DEPTH[IP] + DEPTH[IM]; IZ += 2; }
          }
          IP = klon(ij, 2); IM = klon(ij, 1);
          if (IP != 0 && IM != 0) { D_MEAN = D_MEAN + DEPTH[IP] + DEPTH[IM]; IZ += 2; }
          D_MEAN = D_MEAN / R(IZ);
          IZ = nint_f(std::log(D_MEAN / sh->DEPTHA) / std::log(sh->DEPTHD) + R(1.));
          IZ = std::max(IZ, 1);
          INDEP_G[ij] = std::min(IZ, NDEPTH);
        }
      }
      THDD.assign((size_t)NSEA * KL * ML, 0);
      std::vector<R> TEMP(NSEA + 1, 0);
      if (cfg.shallow_run) {
        for (int k = 1; k <= KL; ++k) {
          for (int ij = 1; ij <= NSEA; ++ij) TEMP[ij] = fd->SINTH[k - 1] * DDPHI[ij] - fd->COSTH[k - 1] * DDLAM[ij];
          for (int m = 1; m <= ML; ++m)
            for (int ij = 1; ij <= NSEA; ++ij) THDD[b(ij, k, m)] = TEMP[ij] * sh->tsihkd(INDEP_G[ij], m - 1);
        }
      }
      if (cfg.shallow_run && cfg.refraction_c_run)
        for (int ij = 1; ij <= NSEA; ++ij) TEMP[ij] = V[ij] * DDPHI[ij] + U[ij] * DDLAM[ij];
      if (cfg.refraction_c_run) {
        SIDC.assign((size_t)NSEA * KL * ML, 0);
        for (int k = 1; k <= KL; ++k) {
          R SS = ipow(fd->SINTH[k - 1], 2), SC = fd->SINTH[k - 1] * fd->COSTH[k - 1], CC = ipow(fd->COSTH[k - 1], 2);
          for (int ij = 1; ij <= NSEA; ++ij) {
            R THDC = SS * DUPHI[ij] + SC * DVPHI[ij] - SC * DULAM[ij] - CC * DVLAM[ij];
            if (cfg.shallow_run) { for (int m = 1; m <= ML; ++m) THDD[b(ij, k, m)] = THDD[b(ij, k, m)] + THDC; }
            else THDD[b(ij, k, ML)] = THDC;
          }
        }
        for (int k = 1; k <= KL; ++k) {
          R SD = fd->SINTH[k - 1], CD = fd->COSTH[k - 1];
          R SS = ipow(SD, 2), SC = SD * CD, CC = ipow(CD, 2);
          for (int ij = 1; ij <= NSEA; ++ij)
            SIDC[b(ij, k, ML)] = -(SC * DUPHI[ij]) - CC * DVPHI[ij] - SS * DULAM[ij] - SC * DVLAM[ij];
        }
        if (cfg.shallow_run) {
          for (int m = 1; m <= ML; ++m)
            for (int k = 1; k <= KL; ++k)
              for (int ij = 1; ij <= NSEA; ++ij)
                SIDC[b(ij, k, m)] = (SIDC[b(ij, k, ML)] * cgond(ij, m) + TEMP[ij] * sh->tsihkd(INDEP_G[ij], m - 1)) *
                                    sh->tfak(INDEP_G[ij], m - 1);
        }
      }
    }
    prepare_coef(THDD, SIDC);
    return check_cfl();
  }

  // PREPARE_PROPAGATION_COEF :837-1913
  void prepare_coef(const std::vector<R>& THDD, const std::vector<R>& SIDC) {
    const bool cur = cfg.refraction_c_run, red = cfg.reduced_grid;
    nic = cur ? 2 : 1; nj = red ? 2 : 1; nlon = cur ? 2 : 1;
    has_sigd = cur;
    has_theta = cfg.spherical_run || cur || (cfg.shallow_run && cfg.refraction_d_run);
    COEF_LAT.assign(nb() * nic * nj, R(0)); COEF_LON.assign(nb() * nlon, R(0)); COEF_SUM.assign(nb(), R(0));
    COEF_THETA.assign(has_theta ? nb() * 2 : 0, R(0)); COEF_SIGD.assign(has_sigd ? nb() * 2 : 0, R(0));
    auto thdd = [&](int ij, int k, int m) { return THDD[b(ij, k, m)]; };
    auto sidc = [&](int ij, int k, int m) { return SIDC[b(ij, k, m)]; };
    const R DELPRO = R(cfg.idelpro);
    std::vector<R> DELLA0(NSEA + 1), DRGM(NSEA + 1), WOK1(NSEA + 1), WOK2(NSEA + 1);
    if (!cfg.spherical_run) {
      if (!cur && !cfg.shallow_run) {  // PREP_CART_DEEP :928-965
        R DELPH0 = DELPRO / DELPHI;
        for (int ij = 1; ij <= NSEA; ++ij) DELLA0[ij] = DELPRO / DELLAM[KFROMIJ[ij - 1] - 1];
        for (int m = 1; m <= ML; ++m)
          for (int k = 1; k <= KL; ++k) {
            R SD = fd->SINTH[k - 1], CD = fd->COSTH[k - 1];
            R DPN = std::fabs(CD * DELPH0 * fd->GOM[m - 1]);
            SD = std::fabs(SD * fd->GOM[m - 1]);
            for (int ij = 1; ij <= NSEA; ++ij) {
              R DLE = SD * DELLA0[ij];
              csum(ij, k, m) = R(1.) - DLE - DPN;
              lon(ij, k, m, 1) = DLE;
              lat(ij, k, m, 1, 1) = DPN;
            }
          }
      } else if (!cur) {  // PREP_CART_SHALLOW :974-1051
        R DELPH0 = R(0.5) * DELPRO / DELPHI, DELTHR = R(0.5) * DELPRO / fd->DELTH;
        for (int ij = 1; ij <= NSEA; ++ij) DELLA0[ij] = R(0.5) * DELPRO / DELLAM[KFROMIJ[ij - 1] - 1];
        for (int m = 1; m <= ML; ++m)
          for (int k = 1; k <= KL; ++k) {
            R SD = std::fabs(fd->SINTH[k - 1]), CD = std::fabs(fd->COSTH[k - 1] * DELPH0);
            int IS = jxo(k, 1), IT = jxo(k, 2), IC = jyo(k, 1), ID = jyo(k, 2);
            for (int ij = 1; ij <= NSEA; ++ij) {
              lon(ij, k, m, 1) = SD * (cgond(klon(ij, IS), m) + cgond(ij, m)) * DELLA0[ij];
              lat(ij, k, m, 1, 1) = CD * (cgond(klat(ij, IC, 1), m) + cgond(ij, m));
              csum(ij, k, m) = R(1.) - SD * (cgond(klon(ij, IT), m) + cgond(ij, m)) * DELLA0[ij] -
                               CD * (cgond(klat(ij, ID, 1), m) + cgond(ij, m));
            }
            if (cfg.refraction_d_run) {
              int KP = kpm(k, 1), KM = kpm(k, -1);
              for (int ij = 1; ij <= NSEA; ++ij) {
                R DTP = (thdd(ij, k, m) + thdd(ij, KP, m)) * DELTHR;
                R DTM = (thdd(ij, k, m) + thdd(ij, KM, m)) * DELTHR;
                csum(ij, k, m) = csum(ij, k, m) - std::max(R(0.), DTP) + std::min(R(0.), DTM);
                theta(ij, k, m, 1) = -std::min(R(0.), DTP);
                theta(ij, k, m, 2) = std::max(R(0.), DTM);
              }
            }
          }
      } else if (!cfg.shallow_run) {  // PREP_CART_DEEP_CUR :1060-1137
        R DELPH0 = R(0.5) * DELPRO / DELPHI, DELTHR = R(0.5) * DELPRO / fd->DELTH;
        R DELFR0 = R(0.5) * DELPRO * R(2.1) / R(0.2);
        for (int ij = 1; ij <= NSEA; ++ij) DELLA0[ij] = R(0.5) * DELPRO / DELLAM[KFROMIJ[ij - 1] - 1];
        for (int m = 1; m <= ML; ++m)
          for (int k = 1; k <= KL; ++k) {
            int KP = kpm(k, 1), KM = kpm(k, -1);
            R CGS = fd->GOM[m - 1] * fd->SINTH[k - 1], CGC = fd->GOM[m - 1] * fd->COSTH[k - 1];
            for (int ij = 0; ij <= NSEA; ++ij) { WOK1[ij] = U[ij] + CGS; WOK2[ij] = (V[ij] + CGC) * DELPH0; }
            for (int ij = 1; ij <= NSEA; ++ij) {
              R DLW = (WOK1[ij] + WOK1[klon(ij, 1)]) * DELLA0[ij];
              R DLE = (WOK1[ij] + WOK1[klon(ij, 2)]) * DELLA0[ij];
              R DTC = R(1.) - std::max(R(0.), DLE) + std::min(R(0.), DLW);
              lon(ij, k, m, 2) = -std::min(R(0.), DLE);
              lon(ij, k, m, 1) = std::max(R(0.), DLW);
              R DPS = WOK2[ij] + WOK2[klat(ij, 1, 1)];
              R DPN = WOK2[ij] + WOK2[klat(ij, 2, 1)];
              DTC = DTC - std::max(R(0.), DPN) + std::min(R(0.), DPS);
              lat(ij, k, m, 2, 1) = -std::min(R(0.), DPN);
              lat(ij, k, m, 1, 1) = std::max(R(0.), DPS);
              R DTP = (thdd(ij, k, ML) + thdd(ij, KP, ML)) * DELTHR;
              R DTM = (thdd(ij, k, ML) + thdd(ij, KM, ML)) * DELTHR;
              DTC = DTC - std::max(R(0.), DTP) + std::min(R(0.), DTM);
              theta(ij, k, m, 1) = -std::min(R(0.), DTP);
              theta(ij, k, m, 2) = std::max(R(0.), DTM);
              R DOM = sidc(ij, k, ML) * DELFR0;
              csum(ij, k, m) = DTC - std::fabs(DOM);
              sigd(ij, k, m, 1) = -std::min(R(0.), DOM) / R(1.1);
              sigd(ij, k, m, 2) = std::max(R(0.), DOM) * R(1.1);
            }
          }
      } else {  // PREP_CART_SHALLOW_CUR :1146-1239
        R DELPH0 = R(0.5) * DELPRO / DELPHI, DELTHR = R(0.5) * DELPRO / fd->DELTH;
        R DELFR0 = R(0.5) * DELPRO / (R(0.1) * C_::ZPI);
        for (int ij = 1; ij <= NSEA; ++ij) DELLA0[ij] = R(0.5) * DELPRO / DELLAM[KFROMIJ[ij - 1] - 1];
        for (int m = 1; m <= ML; ++m) {
          int MM = mpm(m, -1), MP = mpm(m, 1);
          R DFP = DELFR0 / fd->FR[m - 1], DFM = DELFR0 / fd->FR[MM - 1];
          for (int k = 1; k <= KL; ++k) {
            R SD = fd->SINTH[k - 1], CD = fd->COSTH[k - 1];
            int KP = kpm(k, 1), KM = kpm(k, -1);
            for (int ij = 0; ij <= NSEA; ++ij) { WOK1[ij] = U[ij] + SD * cgond(ij, m); WOK2[ij] = (V[ij] + CD * cgond(ij, m)) * DELPH0; }
            for (int ij = 1; ij <= NSEA; ++ij) {
              R DLW = (WOK1[ij] + WOK1[klon(ij, 1)]) * DELLA0[ij];
              R DLE = (WOK1[ij] + WOK1[klon(ij, 2)]) * DELLA0[ij];
              R DTC = R(1.) - std::max(R(0.), DLE) + std::min(R(0.), DLW);
              lon(ij, k, m, 1) = std::max(R(0.), DLW);
              lon(ij, k, m, 2) = -std::min(R(0.), DLE);
              R DPS = WOK2[ij] + WOK2[klat(ij, 1, 1)];
              R DPN = WOK2[ij] + WOK2[klat(ij, 2, 1)];
              DTC = DTC - std::max(R(0.), DPN) + std::min(R(0.), DPS);
              lat(ij, k, m, 1, 1) = std::max(R(0.), DPS);
              lat(ij, k, m, 2, 1) = -std::min(R(0.), DPN);
              R DTP = (thdd(ij, k, m) + thdd(ij, KP, m)) * DELTHR;
              R DTM = (thdd(ij, k, m) + thdd(ij, KM, m)) * DELTHR;
              DTC = DTC - std::max(R(0.), DTP) + std::min(R(0.), DTM);
              theta(ij, k, m, 1) = -std::min(R(0.), DTP);
              theta(ij, k, m, 2) = std::max(R(0.), DTM);
              R DOP = (sidc(ij, k, m) + sidc(ij, k, MP)) * DFP;
              R DOM = (sidc(ij, k, m) + sidc(ij, k, MM)) * DFM;
              sigd(ij, k, m, 1) = -std::min(R(0.), DOP) / R(1.1);
              sigd(ij, k, m, 2) = std::max(R(0.), DOM) * R(1.1);
              csum(ij, k, m) = DTC - std::max(R(0.), DOP) + std::min(R(0.), DOM);
            }
          }
        }
      }
      return;
    }
    // spherical variants
    const R DELTH0 = R(0.5) * DELPRO / fd->DELTR, DELPH0 = R(0.5) * DELPRO / DELPHI, DELTHR = R(0.5) * DELPRO / fd->DELTH;
    for (int ij = 1; ij <= NSEA; ++ij) DRGM[ij] = SINPH[KFROMIJ[ij - 1] - 1] * DCO[ij];
    if (!cur && !cfg.shallow_run) {  // PREP_SPHER_DEEP :1248-1327
      for (int ij = 1; ij <= NSEA; ++ij) DELLA0[ij] = DELPRO * DCO[ij] / DELLAM[KFROMIJ[ij - 1] - 1];
      for (int k = 1; k <= KL; ++k) {
        R SD = fd->SINTH[k - 1], CD = fd->COSTH[k - 1];
        R SDA = std::fabs(SD), CDA = std::fabs(CD * DELPH0);
        int KP = kpm(k, 1), KM = kpm(k, -1), IC = jyo(k, 1), ID = jyo(k, 2);
        R SP = DELTH0 * (fd->SINTH[k - 1] + fd->SINTH[KP - 1]);
        R SM = DELTH0 * (fd->SINTH[k - 1] + fd->SINTH[KM - 1]);
        for (int m = 1; m <= ML; ++m) {
          R GOM = fd->GOM[m - 1];
          for (int ij = 1; ij <= NSEA; ++ij) {
            R DPN = CDA * (dpsn(ij, IC) + R(1.));
            R DLE = SDA * DELLA0[ij];
            R DTC = CDA * (dpsn(ij, ID) + R(1.)) + DLE;
            R DTP = DRGM[ij] * SP, DTM = DRGM[ij] * SM;
            DTC = DTC + std::max(R(0.), DTP) - std::min(R(0.), DTM);
            lat(ij, k, m, 1, 1) = GOM * DPN;
            lon(ij, k, m, 1) = GOM * DLE;
            theta(ij, k, m, 1) = -(GOM * std::min(R(0.), DTP));
            theta(ij, k, m, 2) = GOM * std::max(R(0.), DTM);
            csum(ij, k, m) = R(1.) - GOM * DTC;
          }
          if (red)
            for (int ij = 1; ij <= NSEA; ++ij) {
              lat(ij, k, m, 1, 2) = lat(ij, k, m, 1, 1) * (R(1.) - wlat(ij, IC));
              lat(ij, k, m, 1, 1) = lat(ij, k, m, 1, 1) * wlat(ij, IC);
            }
        }
      }
      return;
    }
    for (int ij = 1; ij <= NSEA; ++ij) DELLA0[ij] = R(0.5) * DELPRO * DCO[ij] / DELLAM[KFROMIJ[ij - 1] - 1];
    if (!cur) {  // PREP_SPHER_SHALLOW :1336-1485
      std::vector<R> CGKLAT((size_t)(NSEA + 1) * ML * 2);
      auto cgk = [&](int ij, int m, int ic) -> R& { return CGKLAT[ij + (size_t)(NSEA + 1) * ((m - 1) + (size_t)ML * (ic - 1))]; };
      for (int ic = 1; ic <= 2; ++ic)
        for (int m = 1; m <= ML; ++m)
          for (int ij = 1; ij <= NSEA; ++ij) {
            if (red)
              cgk(ij, m, ic) = cgond(ij, m) + dpsn(ij, ic) * (wlat(ij, ic) * cgond(klat(ij, ic, 1), m) +
                                                              (R(1.) - wlat(ij, ic)) * cgond(klat(ij, ic, 2), m));
            else cgk(ij, m, ic) = cgond(ij, m) + dpsn(ij, ic) * cgond(klat(ij, ic, 1), m);
          }
      for (int k = 1; k <= KL; ++k) {
        R SD = fd->SINTH[k - 1], CD = fd->COSTH[k - 1];
        R SDA = std::fabs(SD), CDA = std::fabs(CD * DELPH0);
        int KP = kpm(k, 1), KM = kpm(k, -1);
        R SP = DELTH0 * (fd->SINTH[k - 1] + fd->SINTH[KP - 1]);
        R SM = DELTH0 * (fd->SINTH[k - 1] + fd->SINTH[KM - 1]);
        int IS = jxo(k, 1), IT = jxo(k, 2), IC = jyo(k, 1), ID = jyo(k, 2);
        for (int m = 1; m <= ML; ++m)
          for (int ij = 1; ij <= NSEA; ++ij) {
            R DTC = R(1.) - CDA * cgk(ij, m, ID);
            lat(ij, k, m, 1, 1) = CDA * cgk(ij, m, IC);
            DTC = DTC - SDA * (cgond(klon(ij, IT), m) + cgond(ij, m)) * DELLA0[ij];
            lon(ij, k, m, 1) = SDA * (cgond(klon(ij, IS), m) + cgond(ij, m)) * DELLA0[ij];
            R DTP = DRGM[ij] * cgond(ij, m), DTM;
            if (cfg.refraction_d_run) {
              DTM = DTP * SM + (thdd(ij, k, m) + thdd(ij, KM, m)) * DELTHR;
              DTP = DTP * SP + (thdd(ij, k, m) + thdd(ij, KP, m)) * DELTHR;
            } else { DTM = DTP * SM; DTP = DTP * SP; }
            DTC = DTC - std::max(R(0.), DTP) + std::min(R(0.), DTM);
            theta(ij, k, m, 1) = -std::min(R(0.), DTP);
            theta(ij, k, m, 2) = std::max(R(0.), DTM);
            csum(ij, k, m) = DTC;
          }
      }
      if (red)
        for (int m = 1; m <= ML; ++m)
          for (int k = 1; k <= KL; ++k) {
            int IC = jyo(k, 1);
            for (int ij = 1; ij <= NSEA; ++ij) {
              lat(ij, k, m, 1, 2) = lat(ij, k, m, 1, 1) * (R(1.) - wlat(ij, IC));
              lat(ij, k, m, 1, 1) = lat(ij, k, m, 1, 1) * wlat(ij, IC);
            }
          }
      return;
    }
    if (!cfg.shallow_run) {  // PREP_SPHER_DEEP_CURR :1494-1587 and _REG :1591-1676
      const R DELFR0 = R(0.5) * DELPRO * R(2.1) / R(0.2);
      for (int m = 1; m <= ML; ++m)
        for (int k = 1; k <= KL; ++k) {
          R SD = fd->SINTH[k - 1], CD = fd->COSTH[k - 1];
          int KP = kpm(k, 1), KM = kpm(k, -1);
          R GOM = fd->GOM[m - 1];
          R SP = DELTH0 * (fd->SINTH[k - 1] + fd->SINTH[KP - 1]) * GOM;
          R SM = DELTH0 * (fd->SINTH[k - 1] + fd->SINTH[KM - 1]) * GOM;
          R CGS = GOM * SD, CGC = GOM * CD;
          for (int ij = 0; ij <= NSEA; ++ij) { WOK1[ij] = U[ij] + CGS; WOK2[ij] = (V[ij] + CGC) * DELPH0; }
          for (int ij = 1; ij <= NSEA; ++ij) {
            R DLW = (WOK1[ij] + WOK1[klon(ij, 1)]) * DELLA0[ij];
            R DLE = (WOK1[ij] + WOK1[klon(ij, 2)]) * DELLA0[ij];
            R DTC = R(1.) - std::max(R(0.), DLE) + std::min(R(0.), DLW);
            lon(ij, k, m, 2) = -std::min(R(0.), DLE);
            lon(ij, k, m, 1) = std::max(R(0.), DLW);
            if (red) {
              R DPS = (WOK2[ij] + WOK2[klat(ij, 1, 1)] * dpsn(ij, 1)) * wlat(ij, 1);
              R DPS2 = (WOK2[ij] + WOK2[klat(ij, 1, 2)] * dpsn(ij, 1)) * (R(1.) - wlat(ij, 1));
              R DPN = (WOK2[ij] + WOK2[klat(ij, 2, 1)] * dpsn(ij, 2)) * wlat(ij, 2);
              R DPN2 = (WOK2[ij] + WOK2[klat(ij, 2, 2)] * dpsn(ij, 2)) * (R(1.) - wlat(ij, 2));
              DTC = DTC - std::max(R(0.), DPN) - std::max(R(0.), DPN2) + std::min(R(0.), DPS) + std::min(R(0.), DPS2);
              lat(ij, k, m, 2, 1) = -std::min(R(0.), DPN);
              lat(ij, k, m, 2, 2) = -std::min(R(0.), DPN2);
              lat(ij, k, m, 1, 1) = std::max(R(0.), DPS);
              lat(ij, k, m, 1, 2) = std::max(R(0.), DPS2);
            } else {
              R DPS = WOK2[ij] + WOK2[klat(ij, 1, 1)] * dpsn(ij, 1);
              R DPN = WOK2[ij] + WOK2[klat(ij, 2, 1)] * dpsn(ij, 2);
              DTC = DTC - std::max(R(0.), DPN) + std::min(R(0.), DPS);
              lat(ij, k, m, 1, 1) = std::max(R(0.), DPS);
              lat(ij, k, m, 2, 1) = -std::min(R(0.), DPN);
            }
            R DTP = SP * DRGM[ij] + (thdd(ij, k, ML) + thdd(ij, KP, ML)) * DELTHR;
            R DTM = SM * DRGM[ij] + (thdd(ij, k, ML) + thdd(ij, KM, ML)) * DELTHR;
            DTC = DTC - std::max(R(0.), DTP) + std::min(R(0.), DTM);
            theta(ij, k, m, 1) = -std::min(R(0.), DTP);
            theta(ij, k, m, 2) = std::max(R(0.), DTM);
            R DOM = sidc(ij, k, ML) * DELFR0;
            DTC = DTC - std::fabs(DOM);
            sigd(ij, k, m, 1) = -std::min(R(0.), DOM) / R(1.1);
            sigd(ij, k, m, 2) = std::max(R(0.), DOM) * R(1.1);
            csum(ij, k, m) = DTC;
          }
        }
      return;
    }
    {  // PREP_SPHER_SHALLOW_CURR :1685-1804 and _REG :1808-1911
      const R DELFR0 = R(0.5) * DELPRO / (R(0.1) * C_::ZPI);
      for (int m = 1; m <= ML; ++m) {
        int MM = mpm(m, -1), MP = mpm(m, 1);
        R DFP = DELFR0 / fd->FR[m - 1], DFM = DELFR0 / fd->FR[MM - 1];
        for (int k = 1; k <= KL; ++k) {
          R SD = fd->SINTH[k - 1], CD = fd->COSTH[k - 1];
          int KP = kpm(k, 1), KM = kpm(k, -1);
          R SP = DELTH0 * (fd->SINTH[k - 1] + fd->SINTH[KP - 1]);
          R SM = DELTH0 * (fd->SINTH[k - 1] + fd->SINTH[KM - 1]);
          for (int ij = 0; ij <= NSEA; ++ij) { WOK1[ij] = U[ij] + SD * cgond(ij, m); WOK2[ij] = (V[ij] + CD * cgond(ij, m)) * DELPH0; }
          for (int ij = 1; ij <= NSEA; ++ij) {
            R DLW = (WOK1[ij] + WOK1[klon(ij, 1)]) * DELLA0[ij];
            R DLE = (WOK1[ij] + WOK1[klon(ij, 2)]) * DELLA0[ij];
            R DTC = R(1.) - std::max(R(0.), DLE) + std::min(R(0.), DLW);
            lon(ij, k, m, 1) = std::max(R(0.), DLW);
            lon(ij, k, m, 2) = -std::min(R(0.), DLE);
            if (red) {
              R DPS = WOK2[ij] + dpsn(ij, 1) * (wlat(ij, 1) * WOK2[klat(ij, 1, 1)] + (R(1.) - wlat(ij, 1)) * WOK2[klat(ij, 1, 2)]);
              R DPS2 = DPS * (R(1.) - wlat(ij, 1));
              DPS = DPS * wlat(ij, 1);
              R DPN = WOK2[ij] + dpsn(ij, 2) * (wlat(ij, 2) * WOK2[klat(ij, 2, 1)] + (R(1.) - wlat(ij, 2)) * WOK2[klat(ij, 2, 2)]);
              R DPN2 = DPN * (R(1.) - wlat(ij, 2));
              DPN = DPN * wlat(ij, 2);
              DTC = DTC - std::max(R(0.), DPN) - std::max(R(0.), DPN2) + std::min(R(0.), DPS) + std::min(R(0.), DPS2);
              lat(ij, k, m, 1, 1) = std::max(R(0.), DPS);
              lat(ij, k, m, 1, 2) = std::max(R(0.), DPS2);
              lat(ij, k, m, 2, 1) = -std::min(R(0.), DPN);
              lat(ij, k, m, 2, 2) = -std::min(R(0.), DPN2);
            } else {
              R DPS = WOK2[ij] + dpsn(ij, 1) * WOK2[klat(ij, 1, 1)];
              R DPN = WOK2[ij] + dpsn(ij, 2) * WOK2[klat(ij, 2, 1)];
              DTC = DTC - std::max(R(0.), DPN) + std::min(R(0.), DPS);
              lat(ij, k, m, 1, 1) = std::max(R(0.), DPS);
              lat(ij, k, m, 2, 1) = -std::min(R(0.), DPN);
            }
            R DTP = SP * DRGM[ij] * cgond(ij, m) + (thdd(ij, k, m) + thdd(ij, KP, m)) * DELTHR;
            R DTM = SM * DRGM[ij] * cgond(ij, m) + (thdd(ij, k, m) + thdd(ij, KM, m)) * DELTHR;
            DTC = DTC - std::max(R(0.), DTP) + std::min(R(0.), DTM);
            theta(ij, k, m, 1) = -std::min(R(0.), DTP);
            theta(ij, k, m, 2) = std::max(R(0.), DTM);
            R DOP = (sidc(ij, k, m) + sidc(ij, k, MP)) * DFP;
            R DOM = (sidc(ij, k, m) + sidc(ij, k, MM)) * DFM;
            DTC = DTC - std::max(R(0.), DOP) + std::min(R(0.), DOM);
            sigd(ij, k, m, 1) = -std::min(R(0.), DOP) / R(1.1);
            sigd(ij, k, m, 2) = std::max(R(0.), DOM) * R(1.1);
            csum(ij, k, m) = DTC;
          }
        }
      }
    }
  }

  // CHECK_CFL :1917-2138 (single rank). Returns -1 if a coefficient is negative.
  int check_cfl() {
    auto mx = [](const R* p, size_t n) { R v = p[0]; for (size_t i = 1; i < n; ++i) v = std::max(v, p[i]); return v; };
    auto mn = [](const R* p, size_t n) { R v = p[0]; for (size_t i = 1; i < n; ++i) v = std::min(v, p[i]); return v; };
    size_t N = nb();
    R lat11max = mx(COEF_LAT.data(), N * nic), lat11min = mn(COEF_LAT.data(), N * nic);
    R lat12max = R(0.1), lat12min = R(0.1);
    if (cfg.reduced_grid) { lat12max = mx(COEF_LAT.data() + N * nic, N * nic); lat12min = mn(COEF_LAT.data() + N * nic, N * nic); }
    R lon11max = mx(COEF_LON.data(), N), lon11min = mn(COEF_LON.data(), N);
    (void)lon11min;
    R lon12max = R(0.1), lon12min = R(0.1);
    if (cfg.refraction_c_run) { lon12max = mx(COEF_LON.data() + N, N); lon12min = mn(COEF_LON.data() + N, N); }
    R th1max = R(0.1), th1min = R(0.1), th2max = R(0.1), th2min = R(0.1);
    if (has_theta) { th1max = mx(COEF_THETA.data(), N); th1min = mn(COEF_THETA.data(), N); th2max = mx(COEF_THETA.data() + N, N); th2min = mn(COEF_THETA.data() + N, N); }
    R sg1max = R(0.1), sg1min = R(0.1), sg2max = R(0.1), sg2min = R(0.1);
    if (has_sigd) { sg1max = mx(COEF_SIGD.data(), N); sg1min = mn(COEF_SIGD.data(), N); sg2max = mx(COEF_SIGD.data() + N, N); sg2min = mn(COEF_SIGD.data() + N, N); }
    R summax = R(1.) - mn(COEF_SUM.data(), N), summin = R(1.) - mx(COEF_SUM.data(), N);
    R cmax = std::max({lat11max, lat12max, lon11max, lon12max, th1max, th2max, sg1max, sg2max, summax});
    R cmin = std::min({lat11min, lat12min, lon12min, lon12min, th1min, th2min, sg1min, sg2min, summin});
    cfl_min = cmin;
    if (cmin < R(0.)) { total_cfl = cmin; return -1; }
    total_cfl = cmax;
    if (total_cfl > R(0.999)) {
      COUNTER = (int)std::ceil(total_cfl);
      total_cfl = total_cfl / R(COUNTER);
    } else COUNTER = 1;
    if (COUNTER != 1) {
      R c = R(COUNTER);
      for (auto& v : COEF_LAT) v = v / c;
      for (auto& v : COEF_LON) v = v / c;
      for (auto& v : COEF_THETA) v = v / c;
      for (auto& v : COEF_SIGD) v = v / c;
      for (auto& v : COEF_SUM) v = R(1.) - (R(1.) - v) / c;
    }
    return 0;
  }

  // PROPAGS :635-829 on F3[(ij-1) + NSEA*((k-1) + KL*(m-1))]
  // nthreads > 1 spreads the (direction, frequency) planes of each sub-step
  // over host threads; every plane is computed as in the serial loops, so
  // the result does not depend on the thread count.
  void propags(R* F3, int nthreads = 1) {
    std::vector<R> F1((size_t)(NSEA + 1) * KL * ML);
    auto f1 = [&](int ij, int k, int m) -> R& { return F1[ij + (size_t)(NSEA + 1) * ((k - 1) + (size_t)KL * (m - 1))]; };
    auto planes = [&](auto&& fn) {  // fn(k, m) for every plane
      const int n = KL * ML;
      if (nthreads <= 1) { for (int q = 0; q < n; ++q) fn(q % KL + 1, q / KL + 1); return; }
      std::atomic<int> next(0);
      std::vector<std::thread> pool;
      for (int t = 0; t < nthreads; ++t)
        pool.emplace_back([&]() { for (int q; (q = next.fetch_add(1)) < n;) fn(q % KL + 1, q / KL + 1); });
      for (auto& t : pool) t.join();
    };
    for (int it = 0; it < COUNTER; ++it) {
      planes([&](int k, int m) {
        f1(0, k, m) = R(0.);
        for (int ij = 1; ij <= NSEA; ++ij) f1(ij, k, m) = F3[b(ij, k, m)];
      });
      if (cfg.refraction_c_run) {
        planes([&](int k, int m) {
          int MM = mpm(m, -1), MP = mpm(m, 1);
          {
            int KP = kpm(k, 1), KM = kpm(k, -1);
            for (int ij = 1; ij <= NSEA; ++ij) {
              R v = csum(ij, k, m) * f1(ij, k, m) + lat(ij, k, m, 2, 1) * f1(klat(ij, 2, 1), k, m) +
                    lat(ij, k, m, 1, 1) * f1(klat(ij, 1, 1), k, m) + lon(ij, k, m, 2) * f1(klon(ij, 2), k, m) +
                    lon(ij, k, m, 1) * f1(klon(ij, 1), k, m) + theta(ij, k, m, 1) * f1(ij, KP, m) +
                    theta(ij, k, m, 2) * f1(ij, KM, m) + sigd(ij, k, m, 1) * f1(ij, k, MP) + sigd(ij, k, m, 2) * f1(ij, k, MM);
              if (cfg.reduced_grid)
                v = v + lat(ij, k, m, 2, 2) * f1(klat(ij, 2, 2), k, m) + lat(ij, k, m, 1, 2) * f1(klat(ij, 1, 2), k, m);
              F3[b(ij, k, m)] = v;
            }
          }
        });
      } else {
        planes([&](int k, int m) {
          int KP = kpm(k, 1), KM = kpm(k, -1), IS = jxo(k, 1), IC = jyo(k, 1);
          {
            for (int ij = 1; ij <= NSEA; ++ij) {
              R v = csum(ij, k, m) * f1(ij, k, m) + lat(ij, k, m, 1, 1) * f1(klat(ij, IC, 1), k, m) +
                    lon(ij, k, m, 1) * f1(klon(ij, IS), k, m);
              if (cfg.refraction_d_run || cfg.spherical_run)
                v = v + theta(ij, k, m, 1) * f1(ij, KP, m) + theta(ij, k, m, 2) * f1(ij, KM, m);
              if (cfg.reduced_grid) v = v + lat(ij, k, m, 1, 2) * f1(klat(ij, IC, 2), k, m);
              F3[b(ij, k, m)] = v;
            }
          }
        });
      }
    }
  }
};

}  // namespace wamo
