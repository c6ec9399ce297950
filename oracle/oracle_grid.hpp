// ORACLE — test infrastructure only (see oracle_tables.hpp header).
//
// Restatement of the reference grid tooling that produces the propagation
// neighbour tables: PREPARE_GRID geometry (preproc_module.f90:2128-2193),
// the sea-point numbering and KLAT/KLON/WLAT builder (:2285-2363),
// CLOSEST_GP_LAT (:1318-1484), and the cosine-of-latitude factors DCO/DPSN
// (wam_initial_module.f90:204-214).
#pragma once
#include "oracle_tables.hpp"

namespace wamo {

struct GridDef {
  int NX, NY;
  int AMOSOP, AMOWEP, AMOEAP, XDELLA, XDELLO;  // [M_SEC] = 1/100 arc-second
  int reduced_grid;
};
constexpr int M_DEGREE = 60 * 60 * 100;          // wam_coordinate_module.f90:41-43
constexpr int M_S_PER = 360 * M_DEGREE;

template <typename R> struct Grid {
  int NX, NY, NSEA; bool IPER;
  R DELPHI;
  std::vector<int> NLON_RG, ZDELLO;
  std::vector<R> SINPH, COSPH, DELLAM;      // per latitude row (1..NY at [k-1])
  std::vector<int> IXLG, KXLT;              // per sea point, 1-based values
  std::vector<int> KLAT;                    // [(ip-1) + NSEA*((ic-1) + 2*(j-1))], 0 = land
  std::vector<int> KLON;                    // [(ip-1) + NSEA*(i-1)]
  std::vector<R> WLAT;                      // [(ip-1) + NSEA*(ic-1)]
  std::vector<int> KFROMIJ;                 // 1-based latitude row per sea point

  // mask[(i-1) + NX*(k-1)] != 0 means sea
  void build(const GridDef& g, const std::vector<uint8_t>& mask) {
    using C_ = K<R>;
    NX = g.NX; NY = g.NY;
    SINPH.resize(NY); COSPH.resize(NY);
    for (int k = 1; k <= NY; ++k) {                                   // :2131-2135
      R XLAT = R(g.AMOSOP + (k - 1) * g.XDELLA) / R(M_DEGREE) * C_::RAD;
      SINPH[k - 1] = std::sin(XLAT); COSPH[k - 1] = std::cos(XLAT);
    }
    DELPHI = R(g.XDELLA) / R(M_DEGREE) * C_::CIRC / R(360.);          // :2142
    NLON_RG.assign(NY, NX);
    if (g.reduced_grid) {                                             // :2146-2149
      R cmax = *std::max_element(COSPH.begin(), COSPH.end());
      for (int k = 0; k < NY; ++k) {
        int n = nint_f(R(NX) * COSPH[k] / cmax);
        if (n % 2 == 1) n += 1;
        NLON_RG[k] = std::min(n, NX);
      }
    }
    // periodicity: wam_coordinate_module.f90:706-746, called at preproc_module.f90:536
    IPER = std::abs(g.AMOWEP - g.AMOEAP - g.XDELLO + M_S_PER) <= NX / 2;
    ZDELLO.resize(NY); DELLAM.resize(NY);
    for (int k = 0; k < NY; ++k) {                                    // :2187-2193
      if (IPER) ZDELLO[k] = nint_f(R(g.AMOEAP - g.AMOWEP + g.XDELLO) / R(NLON_RG[k]));
      else ZDELLO[k] = nint_f(R(g.AMOEAP - g.AMOWEP) / R(NLON_RG[k] - 1));
      DELLAM[k] = R(ZDELLO[k]) / R(M_DEGREE) * C_::CIRC / R(360.);
    }
    auto sea = [&](int i, int k) { return mask[(i - 1) + (size_t)NX * (k - 1)] != 0; };
    // :2288-2297
    IXLG.clear(); KXLT.clear();
    for (int k = 1; k <= NY; ++k)
      for (int i = 1; i <= NX; ++i)
        if (sea(i, k)) { IXLG.push_back(i); KXLT.push_back(k); }
    NSEA = (int)IXLG.size();
    KLAT.assign((size_t)NSEA * 4, 0); KLON.assign((size_t)NSEA * 2, 0); WLAT.assign((size_t)NSEA * 2, 0);
    KFROMIJ = KXLT;
    auto count_row = [&](int k, int i0, int i1) { int c = 0; for (int i = i0; i <= i1; ++i) c += sea(i, k); return c; };
    for (int ip = 1; ip <= NSEA; ++ip) {                              // :2320-2363
      int i = IXLG[ip - 1], k = KXLT[ip - 1];
      if (i > 1) { if (sea(i - 1, k)) KLON[(ip - 1)] = ip - 1; }
      else { if (IPER && sea(NLON_RG[k - 1], k)) KLON[(ip - 1)] = ip + count_row(k, 2, NX); }
      if (i < NLON_RG[k - 1]) { if (sea(i + 1, k)) KLON[(ip - 1) + NSEA] = ip + 1; }
      else { if (IPER && sea(1, k)) KLON[(ip - 1) + NSEA] = ip + 1 - count_row(k, 1, NX); }
      for (int ic = 1; ic <= 2; ++ic) {
        int kh = (ic == 1) ? k - 1 : k + 1;
        int ip1 = 0, ip2 = 0; R wh = R(1);
        if ((ic == 1 && k > 1) || (ic == 2 && k < NY)) {
          R XH = R(i - 1) * R(ZDELLO[k - 1]) / R(ZDELLO[kh - 1]);
          closest_gp_lat(mask, i, k, ip, XH, kh, ip1, ip2, wh);
        }
        KLAT[(ip - 1) + NSEA * ((ic - 1) + 2 * 0)] = ip1;
        KLAT[(ip - 1) + NSEA * ((ic - 1) + 2 * 1)] = ip2;
        WLAT[(ip - 1) + NSEA * (ic - 1)] = wh;
      }
    }
  }

  void closest_gp_lat(const std::vector<uint8_t>& mask, int I, int Kr, int IP, R XH, int KH, int& IP1, int& IP2, R& WH) {
    auto sea = [&](int i, int k) { return mask[(i - 1) + (size_t)NX * (k - 1)] != 0; };
    WH = R(1.); IP1 = 0; IP2 = 0;
    int ICA, ICE, ICS;
    if (KH < Kr) { if (KH < 1) return; ICA = IP; ICE = 1; ICS = -1; }
    else { if (KH > NY) return; ICA = IP; ICE = NSEA; ICS = +1; }
    int IPH1, IPH2;
    if (NLON_RG[KH - 1] == NLON_RG[Kr - 1]) { IPH1 = I; IPH2 = I; }
    else {
      IPH1 = (int)std::floor(XH); IPH2 = (int)std::ceil(XH);
      if (IPH1 == IPH2) { IPH1 = IPH1 + 1; IPH2 = IPH1; }
      else if (IPH2 == nint_f(XH)) { int IPH = IPH1; IPH1 = IPH2 + 1; IPH2 = IPH + 1; }
      else { IPH1 = IPH1 + 1; IPH2 = IPH2 + 1; }
    }
    if (IPH1 != IPH2) {                                               // :1424-1434
      R Z = R(ZDELLO[KH - 1]) / R(ZDELLO[Kr - 1]);
      R D3 = XH * Z - R(0.5), D5 = XH * Z + R(0.5);
      R XP = R(IPH1 - 1) * Z;
      R D4 = XP - R(0.5) * Z, D6 = XP + R(0.5) * Z;
      if (D4 < D3 || D6 > D5) WH = std::min(R(1.), std::min(D5, D6) - std::max(D3, D4));
    }
    auto search = [&](int iph) {
      int IC = ICA;
      for (IC = ICA; ICS > 0 ? IC <= ICE : IC >= ICE; IC += ICS)
        if (IXLG[IC - 1] == iph && KXLT[IC - 1] == KH) break;
      return IC;
    };
    if (IPER) {
      if (IPH1 < 1) IPH1 += NLON_RG[KH - 1];
      if (IPH1 > NLON_RG[KH - 1]) IPH1 -= NLON_RG[KH - 1];
    }
    if (IPH1 >= 1 && IPH1 <= NLON_RG[KH - 1] && sea(IPH1, KH)) IP1 = search(IPH1);
    if (IPH1 != IPH2) {
      if (IPER) {
        if (IPH2 < 1) IPH2 += NLON_RG[KH - 1];
        if (IPH2 > NLON_RG[KH - 1]) IPH2 -= NLON_RG[KH - 1];
      }
      if (IPH2 >= 1 && IPH2 <= NLON_RG[KH - 1] && sea(IPH2, KH)) IP2 = search(IPH2);
    } else IP2 = IP1;
  }
};

}  // namespace wamo
