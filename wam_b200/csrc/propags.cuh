// PROPAGS on sm_100a.  The reference precomputes four to nine propagation
// coefficient arrays of the full spectrum size in PREPARE_PROPAGATION_COEF
// (wam_propagation_module.f90:837-1913) and streams them in every sub-step;
// here the coefficients are recomputed inside the stencil from a handful of
// per-point metadata (depth-table indices, gradients, metric factors), so a
// sub-step moves only the spectrum itself: one read and one write per bin.
//
// Thread layout: one thread per (sea point, frequency), looping over the
// directions; the direction neighbours K+-1 needed by the refraction terms are
// kept in a register window.  Consecutive threads handle consecutive sea
// points, so every access to FL3(IJ,K,M) is coalesced; the north/south
// neighbours of a latitude row are re-read from L2.
//
// Direction sines and cosines travel in the metadata block itself (a
// __grid_constant__ kernel parameter), so grids with different KL can live
// side by side in one process.
//
// The coefficient formulas keep the reference's operation order and are
// compiled without FMA contraction, so they reproduce the reference's REAL
// coefficients.  Routine map: PREP_CART_DEEP :928, PREP_CART_SHALLOW :974,
// PREP_CART_DEEP_CUR :1060, PREP_CART_SHALLOW_CUR :1146, PREP_SPHER_DEEP
// :1248, PREP_SPHER_SHALLOW :1336, PREP_SPHER_DEEP_CURR(_REG) :1494/:1591,
// PREP_SPHER_SHALLOW_CURR(_REG) :1685/:1808, CHECK_CFL rescaling :2126-2134,
// PROP_NO_CURR :750-785, PROP_CURR :794-825.
#pragma once
#include <cstdint>
#include "wamgpu_config.hpp"
#include "devmath.cuh"
#include "propargs.hpp"

namespace wamgpu {

template <typename R> struct Coefs {
  R sum, lat11, lat21, lat12, lat22, lon1, lon2, th1, th2, sg1, sg2;
};

constexpr bool var_shallow(int v) { return v == V_CART_SHALLOW || v == V_SPHER_SHALLOW || v == V_CART_SHALLOW_CUR || v == V_SPHER_SHALLOW_CURR; }
constexpr bool var_current(int v) { return v == V_CART_DEEP_CUR || v == V_SPHER_DEEP_CURR || v == V_CART_SHALLOW_CUR || v == V_SPHER_SHALLOW_CURR; }
constexpr bool var_spher(int v) { return v >= V_SPHER_DEEP; }

// Everything about sea point i at frequency m that does not depend on the
// direction, loaded once; coef(k) then evaluates the reference's coefficient
// expressions for one direction.
template <typename R, int VAR, bool RED, bool REFRD> struct Site {
  static constexpr bool SH = var_shallow(VAR), CUR = var_current(VAR), SPH = var_spher(VAR);
  const PropArgs<R>& A;
  int i, m, s0, n0, w0, e0, s1, n1;
  R gom, cg, cgS, cgN, cgW, cgE, cgS1, cgN1, d0, dr, ps, pn, wl1, wl2, tsi, ddphi, ddlam;
  R duphi, dulam, dvphi, dvlam, u0, uW, uE, v0, vS, vN, vS1, vN1;
  R dfp, dfm, cgP, cgM, tsiP, tsiM, tfk, tfkP, tfkM, tempc;
  int mp, mm;

  __device__ R cgond(int p1, int mm_) const {
    int jd = (p1 == 0) ? A.NDEPTH : __ldg(&A.indep[p1 - 1]);
    return __ldg(&A.TCGOND[(jd - 1) + A.NDEPTH * mm_]);
  }
  __device__ R uv(const R* f, int p1) const { return p1 == 0 ? R(0) : __ldg(&f[p1 - 1]); }

  __device__ R dir_sin(int k) const { return A.sinth[k]; }
  __device__ R dir_cos(int k) const { return A.costh[k]; }

  __device__ Site(const PropArgs<R>& a, int i_, int m_) : A(a), i(i_), m(m_) {
    const int ns = A.nsea;
    s0 = __ldg(&A.klat[i]); n0 = __ldg(&A.klat[i + ns]);
    w0 = __ldg(&A.klon[i]); e0 = __ldg(&A.klon[i + ns]);
    s1 = RED ? __ldg(&A.klat[i + 2 * ns]) : 0; n1 = RED ? __ldg(&A.klat[i + 3 * ns]) : 0;
    gom = __ldg(&A.GOM[m]);
    d0 = __ldg(&A.della0[i]);
    dr = SPH ? __ldg(&A.drgm[i]) : R(0);
    ps = SPH ? __ldg(&A.dpsn[i]) : R(1); pn = SPH ? __ldg(&A.dpsn[i + ns]) : R(1);
    wl1 = RED ? __ldg(&A.wlat[i]) : R(1); wl2 = RED ? __ldg(&A.wlat[i + ns]) : R(1);
    if (SH) {
      cg = cgond(i + 1, m); cgS = cgond(s0, m); cgN = cgond(n0, m); cgW = cgond(w0, m); cgE = cgond(e0, m);
      cgS1 = RED ? cgond(s1, m) : R(0); cgN1 = RED ? cgond(n1, m) : R(0);
    }
    if (SH && (REFRD || CUR)) {
      int ig = __ldg(&A.indep_g[i]);
      tsi = __ldg(&A.TSIHKD[(ig - 1) + A.NDEPTH * m]);
      ddphi = __ldg(&A.ddphi[i]); ddlam = __ldg(&A.ddlam[i]);
    }
    if (CUR) {
      duphi = __ldg(&A.duphi[i]); dulam = __ldg(&A.dulam[i]); dvphi = __ldg(&A.dvphi[i]); dvlam = __ldg(&A.dvlam[i]);
      u0 = uv(A.u, i + 1); uW = uv(A.u, w0); uE = uv(A.u, e0);
      v0 = uv(A.v, i + 1); vS = uv(A.v, s0); vN = uv(A.v, n0);
      vS1 = RED ? uv(A.v, s1) : R(0); vN1 = RED ? uv(A.v, n1) : R(0);
      if (SH) {
        mm = (m == 0) ? 0 : m - 1; mp = (m == A.ML - 1) ? A.ML - 1 : m + 1;
        dfp = A.DELFR0 / __ldg(&A.FR[m]); dfm = A.DELFR0 / __ldg(&A.FR[mm]);
        int ig = __ldg(&A.indep_g[i]);
        cgP = cgond(i + 1, mp); cgM = cgond(i + 1, mm);
        tsiP = __ldg(&A.TSIHKD[(ig - 1) + A.NDEPTH * mp]); tsiM = __ldg(&A.TSIHKD[(ig - 1) + A.NDEPTH * mm]);
        tfk = __ldg(&A.TFAK[(ig - 1) + A.NDEPTH * m]); tfkP = __ldg(&A.TFAK[(ig - 1) + A.NDEPTH * mp]);
        tfkM = __ldg(&A.TFAK[(ig - 1) + A.NDEPTH * mm]);
        tempc = __ldg(&A.v[i]) * ddphi + __ldg(&A.u[i]) * ddlam;
      }
    }
  }

  // THDD(i,k,m): depth part (PREPARE_PROPAGATION :482-492) plus current part (:521-536)
  __device__ R thdd(int k) const { return thdd_sc(dir_sin(k), dir_cos(k)); }
  __device__ R thdd_sc(R sn, R cs) const {
    R t = R(0);
    if (SH) t = (sn * ddphi - cs * ddlam) * tsi;
    if (CUR) {
      R ss = sn * sn, sc = sn * cs, cc = cs * cs;
      R thdc = ss * duphi + sc * dvphi - sc * dulam - cc * dvlam;
      t = SH ? t + thdc : thdc;
    }
    return t;
  }
  // SIDC(i,k,m') for m' = m, mp, mm (:541-563)
  __device__ R sidc_base_sc(R sd, R cd) const {
    R ss = sd * sd, sc = sd * cd, cc = cd * cd;
    return -(sc * duphi) - cc * dvphi - ss * dulam - sc * dvlam;
  }

  // Direction-dependent inputs of the coefficients of direction k: sines and
  // cosines of k and its neighbours and THDD of k-1, k, k+1.  The stencil loop
  // slides this window along the directions instead of re-reading them.
  struct Win { R sn, cs, snp, csp, snm, th0, thp, thm; };
  static constexpr bool NEED_TH = (SH && REFRD) || CUR;
  __device__ Win window(int k) const {
    const int KL = A.KL;
    const int kp = (k + 1 == KL) ? 0 : k + 1, km = (k == 0) ? KL - 1 : k - 1;
    Win w;
    w.sn = dir_sin(k); w.cs = dir_cos(k);
    w.snp = dir_sin(kp); w.csp = dir_cos(kp);
    w.snm = dir_sin(km);
    if (NEED_TH) { w.th0 = thdd_sc(w.sn, w.cs); w.thp = thdd_sc(w.snp, w.csp); w.thm = thdd(km); }
    else { w.th0 = w.thp = w.thm = R(0); }
    return w;
  }
  // the window of direction k+1 from that of k
  __device__ void advance(Win& w, int k) const {
    const int KL = A.KL;
    const int kpp = (k + 2 >= KL) ? k + 2 - KL : k + 2;
    w.snm = w.sn; w.sn = w.snp; w.cs = w.csp;
    w.snp = dir_sin(kpp); w.csp = dir_cos(kpp);
    if (NEED_TH) { w.thm = w.th0; w.th0 = w.thp; w.thp = thdd_sc(w.snp, w.csp); }
  }
  __device__ Coefs<R> coef(int k) const { return coef_w(window(k)); }

  __device__ Coefs<R> coef_w(const Win& W) const {
    Coefs<R> c = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const R sn = W.sn, cs = W.cs;
    const bool IS0 = sn >= R(0.), IC0 = cs >= R(0.);
    const R z = R(0.);
    if (VAR == V_CART_DEEP) {
      R dpn = dabs(cs * A.DELPH0 * gom);
      R sd = dabs(sn * gom);
      R dle = sd * d0;
      c.sum = R(1.) - dle - dpn; c.lon1 = dle; c.lat11 = dpn;
    } else if (VAR == V_CART_SHALLOW) {
      R sd = dabs(sn), cd = dabs(cs * A.DELPH0);
      c.lon1 = sd * ((IS0 ? cgW : cgE) + cg) * d0;
      c.lat11 = cd * ((IC0 ? cgS : cgN) + cg);
      c.sum = R(1.) - sd * ((IS0 ? cgE : cgW) + cg) * d0 - cd * ((IC0 ? cgN : cgS) + cg);
      if (REFRD) {
        R t0 = W.th0;
        R dtp = (t0 + W.thp) * A.DELTHR, dtm = (t0 + W.thm) * A.DELTHR;
        c.sum = c.sum - dmax(z, dtp) + dmin(z, dtm);
        c.th1 = -dmin(z, dtp); c.th2 = dmax(z, dtm);
      }
    } else if (VAR == V_SPHER_DEEP) {
      R sda = dabs(sn), cda = dabs(cs * A.DELPH0);
      R sp = A.DELTH0 * (sn + W.snp), sm = A.DELTH0 * (sn + W.snm);
      R dpn = cda * ((IC0 ? ps : pn) + R(1.));
      R dle = sda * d0;
      R dtc = cda * ((IC0 ? pn : ps) + R(1.)) + dle;
      R dtp = dr * sp, dtm = dr * sm;
      dtc = dtc + dmax(z, dtp) - dmin(z, dtm);
      c.lat11 = gom * dpn; c.lon1 = gom * dle;
      c.th1 = -(gom * dmin(z, dtp)); c.th2 = gom * dmax(z, dtm);
      c.sum = R(1.) - gom * dtc;
      if (RED) { R wl = IC0 ? wl1 : wl2; c.lat12 = c.lat11 * (R(1.) - wl); c.lat11 = c.lat11 * wl; }
    } else if (VAR == V_SPHER_SHALLOW) {
      R sda = dabs(sn), cda = dabs(cs * A.DELPH0);
      R sp = A.DELTH0 * (sn + W.snp), sm = A.DELTH0 * (sn + W.snm);
      R cgk1, cgk2;  // CGKLAT(IJ,M,1) south and (IJ,M,2) north
      if (RED) {
        cgk1 = cg + ps * (wl1 * cgS + (R(1.) - wl1) * cgS1);
        cgk2 = cg + pn * (wl2 * cgN + (R(1.) - wl2) * cgN1);
      } else { cgk1 = cg + ps * cgS; cgk2 = cg + pn * cgN; }
      R dtc = R(1.) - cda * (IC0 ? cgk2 : cgk1);
      c.lat11 = cda * (IC0 ? cgk1 : cgk2);
      dtc = dtc - sda * ((IS0 ? cgE : cgW) + cg) * d0;
      c.lon1 = sda * ((IS0 ? cgW : cgE) + cg) * d0;
      R dtp = dr * cg, dtm;
      if (REFRD) {
        R t0 = W.th0;
        dtm = dtp * sm + (t0 + W.thm) * A.DELTHR;
        dtp = dtp * sp + (t0 + W.thp) * A.DELTHR;
      } else { dtm = dtp * sm; dtp = dtp * sp; }
      dtc = dtc - dmax(z, dtp) + dmin(z, dtm);
      c.th1 = -dmin(z, dtp); c.th2 = dmax(z, dtm);
      c.sum = dtc;
      if (RED) { R wl = IC0 ? wl1 : wl2; c.lat12 = c.lat11 * (R(1.) - wl); c.lat11 = c.lat11 * wl; }
    } else if (VAR == V_CART_DEEP_CUR || VAR == V_SPHER_DEEP_CURR) {
      R cgs = gom * sn, cgc = gom * cs;
      R w1 = u0 + cgs, w2 = (v0 + cgc) * A.DELPH0;
      R dlw = (w1 + (uW + cgs)) * d0, dle = (w1 + (uE + cgs)) * d0;
      R dtc = R(1.) - dmax(z, dle) + dmin(z, dlw);
      c.lon2 = -dmin(z, dle); c.lon1 = dmax(z, dlw);
      auto wok2 = [&](R vv) { return (vv + cgc) * A.DELPH0; };
      if (!SPH) {
        R dps = w2 + wok2(vS), dpn = w2 + wok2(vN);
        dtc = dtc - dmax(z, dpn) + dmin(z, dps);
        c.lat21 = -dmin(z, dpn); c.lat11 = dmax(z, dps);
      } else if (RED) {
        R dps = (w2 + wok2(vS) * ps) * wl1, dps2 = (w2 + wok2(vS1) * ps) * (R(1.) - wl1);
        R dpn = (w2 + wok2(vN) * pn) * wl2, dpn2 = (w2 + wok2(vN1) * pn) * (R(1.) - wl2);
        dtc = dtc - dmax(z, dpn) - dmax(z, dpn2) + dmin(z, dps) + dmin(z, dps2);
        c.lat21 = -dmin(z, dpn); c.lat22 = -dmin(z, dpn2); c.lat11 = dmax(z, dps); c.lat12 = dmax(z, dps2);
      } else {
        R dps = w2 + wok2(vS) * ps, dpn = w2 + wok2(vN) * pn;
        dtc = dtc - dmax(z, dpn) + dmin(z, dps);
        c.lat11 = dmax(z, dps); c.lat21 = -dmin(z, dpn);
      }
      R t0 = W.th0, tp = W.thp, tm = W.thm;
      R dtp, dtm;
      if (SPH) {
        R sp = A.DELTH0 * (sn + W.snp) * gom, sm = A.DELTH0 * (sn + W.snm) * gom;
        dtp = sp * dr + (t0 + tp) * A.DELTHR; dtm = sm * dr + (t0 + tm) * A.DELTHR;
      } else { dtp = (t0 + tp) * A.DELTHR; dtm = (t0 + tm) * A.DELTHR; }
      dtc = dtc - dmax(z, dtp) + dmin(z, dtm);
      c.th1 = -dmin(z, dtp); c.th2 = dmax(z, dtm);
      R dom = sidc_base_sc(sn, cs) * A.DELFR0;
      c.sum = dtc - dabs(dom);
      c.sg1 = -dmin(z, dom) / R(1.1); c.sg2 = dmax(z, dom) * R(1.1);
    } else {  // V_CART_SHALLOW_CUR, V_SPHER_SHALLOW_CURR
      R w1 = u0 + sn * cg, w2 = (v0 + cs * cg) * A.DELPH0;
      R dlw = (w1 + (uW + sn * cgW)) * d0, dle = (w1 + (uE + sn * cgE)) * d0;
      R dtc = R(1.) - dmax(z, dle) + dmin(z, dlw);
      c.lon1 = dmax(z, dlw); c.lon2 = -dmin(z, dle);
      auto wok2 = [&](R vv, R cgv) { return (vv + cs * cgv) * A.DELPH0; };
      if (!SPH) {
        R dps = w2 + wok2(vS, cgS), dpn = w2 + wok2(vN, cgN);
        dtc = dtc - dmax(z, dpn) + dmin(z, dps);
        c.lat11 = dmax(z, dps); c.lat21 = -dmin(z, dpn);
      } else if (RED) {
        R dps = w2 + ps * (wl1 * wok2(vS, cgS) + (R(1.) - wl1) * wok2(vS1, cgS1));
        R dps2 = dps * (R(1.) - wl1); dps = dps * wl1;
        R dpn = w2 + pn * (wl2 * wok2(vN, cgN) + (R(1.) - wl2) * wok2(vN1, cgN1));
        R dpn2 = dpn * (R(1.) - wl2); dpn = dpn * wl2;
        dtc = dtc - dmax(z, dpn) - dmax(z, dpn2) + dmin(z, dps) + dmin(z, dps2);
        c.lat11 = dmax(z, dps); c.lat12 = dmax(z, dps2); c.lat21 = -dmin(z, dpn); c.lat22 = -dmin(z, dpn2);
      } else {
        R dps = w2 + ps * wok2(vS, cgS), dpn = w2 + pn * wok2(vN, cgN);
        dtc = dtc - dmax(z, dpn) + dmin(z, dps);
        c.lat11 = dmax(z, dps); c.lat21 = -dmin(z, dpn);
      }
      R t0 = W.th0, tp = W.thp, tm = W.thm;
      R dtp, dtm;
      if (SPH) {
        R sp = A.DELTH0 * (sn + W.snp), sm = A.DELTH0 * (sn + W.snm);
        dtp = sp * dr * cg + (t0 + tp) * A.DELTHR; dtm = sm * dr * cg + (t0 + tm) * A.DELTHR;
      } else { dtp = (t0 + tp) * A.DELTHR; dtm = (t0 + tm) * A.DELTHR; }
      dtc = dtc - dmax(z, dtp) + dmin(z, dtm);
      c.th1 = -dmin(z, dtp); c.th2 = dmax(z, dtm);
      R b = sidc_base_sc(sn, cs);
      R s0v = (b * cg + tempc * tsi) * tfk, sPv = (b * cgP + tempc * tsiP) * tfkP, sMv = (b * cgM + tempc * tsiM) * tfkM;
      R dop = (s0v + sPv) * dfp, dom = (s0v + sMv) * dfm;
      c.sg1 = -dmin(z, dop) / R(1.1); c.sg2 = dmax(z, dom) * R(1.1);
      c.sum = dtc - dmax(z, dop) + dmin(z, dom);
    }
    if (A.counter != 1) {  // CHECK_CFL sub-stepping rescale :2126-2134
      const R rc = A.rcounter;
      c.lat11 = c.lat11 / rc; c.lat21 = c.lat21 / rc; c.lat12 = c.lat12 / rc; c.lat22 = c.lat22 / rc;
      c.lon1 = c.lon1 / rc; c.lon2 = c.lon2 / rc; c.th1 = c.th1 / rc; c.th2 = c.th2 / rc;
      c.sg1 = c.sg1 / rc; c.sg2 = c.sg2 / rc;
      c.sum = R(1.) - (R(1.) - c.sum) / rc;
    }
    return c;
  }
};

}  // namespace wamgpu
