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

namespace wamgpu {

enum PropVariant : int {
  V_CART_DEEP = 0, V_CART_SHALLOW = 1, V_CART_DEEP_CUR = 2, V_CART_SHALLOW_CUR = 3,
  V_SPHER_DEEP = 4, V_SPHER_SHALLOW = 5, V_SPHER_DEEP_CURR = 6, V_SPHER_SHALLOW_CURR = 7
};

// Per-sea-point metadata (index i = 0-based local point; neighbour values are
// 1-based local numbers, 0 = land).  Arrays are of length n_ext (local points
// followed by halo points) unless noted.
template <typename R> struct PropArgs {
  int nsea, ld, KL, ML, variant, reduced, refr_d, spherical, counter, NDEPTH;
  R DELPH0, DELTH0, DELTHR, DELFR0, rcounter;
  const int* klat;    // [i + nsea*(ic + 2*j)]   (nsea entries per slot)
  const int* klon;    // [i + nsea*dir]
  const R* wlat;      // [i + nsea*ic]
  const R* dpsn;      // [i + nsea*ic]
  const R* della0;    // [i]   (variant-specific longitude metric factor)
  const R* drgm;      // [i]   SINPH*DCO
  const int* indep;   // [n_ext] depth-table index (1-based), CGOND of point and neighbours
  const int* indep_g; // [i]   averaged depth index for refraction
  const R* ddphi;     // [i]   depth gradients (DDLAM already times DCO on spherical grids)
  const R* ddlam;
  const R* duphi; const R* dulam; const R* dvphi; const R* dvlam;  // current gradients
  const R* u; const R* v;    // [n_ext] currents (land slot reads as 0)
  const R* TCGOND; const R* TSIHKD; const R* TFAK;  // depth tables [(jd-1) + NDEPTH*m]
  const R* GOM; const R* FR; const R* SINTH; const R* COSTH;  // small tables (global)
};

template <typename R> struct Coefs {
  R sum, lat11, lat21, lat12, lat22, lon1, lon2, th1, th2, sg1, sg2;
};

template <typename R> struct PropCore {
  const PropArgs<R>& A;
  __device__ explicit PropCore(const PropArgs<R>& a) : A(a) {}
  __device__ int klat(int i, int ic, int j) const { return __ldg(&A.klat[i + A.nsea * (ic + 2 * j)]); }
  __device__ int klon(int i, int d) const { return __ldg(&A.klon[i + A.nsea * d]); }
  // CGOND of a 1-based local point (0 = land slot: deepest table entry)
  __device__ R cgond(int p1, int m) const {
    int jd = (p1 == 0) ? A.NDEPTH : __ldg(&A.indep[p1 - 1]);
    return __ldg(&A.TCGOND[(jd - 1) + A.NDEPTH * m]);
  }
  __device__ R uv(const R* f, int p1) const { return p1 == 0 ? R(0) : __ldg(&f[p1 - 1]); }

  // depth-refraction turning rate THDD(i,k,m) (PREPARE_PROPAGATION :482-492)
  // plus the current part THDC (:521-536)
  __device__ R thdd(int i, int k, int m, R tsihkd_g) const {
    R t = 0;
    if (A.variant == V_CART_SHALLOW || A.variant == V_SPHER_SHALLOW || A.variant == V_CART_SHALLOW_CUR ||
        A.variant == V_SPHER_SHALLOW_CURR) {
      R temp = __ldg(&A.SINTH[k]) * __ldg(&A.ddphi[i]) - __ldg(&A.COSTH[k]) * __ldg(&A.ddlam[i]);
      t = temp * tsihkd_g;
    }
    if (A.variant == V_CART_DEEP_CUR || A.variant == V_SPHER_DEEP_CURR || A.variant == V_CART_SHALLOW_CUR ||
        A.variant == V_SPHER_SHALLOW_CURR) {
      R sn = __ldg(&A.SINTH[k]), cs = __ldg(&A.COSTH[k]);
      R ss = sn * sn, sc = sn * cs, cc = cs * cs;
      R thdc = ss * __ldg(&A.duphi[i]) + sc * __ldg(&A.dvphi[i]) - sc * __ldg(&A.dulam[i]) - cc * __ldg(&A.dvlam[i]);
      t = (A.variant == V_CART_DEEP_CUR || A.variant == V_SPHER_DEEP_CURR) ? thdc : t + thdc;
    }
    return t;
  }
  // frequency shifting rate SIDC(i,k,m) (PREPARE_PROPAGATION :541-563)
  __device__ R sidc(int i, int k, int m) const {
    R sd = __ldg(&A.SINTH[k]), cd = __ldg(&A.COSTH[k]);
    R ss = sd * sd, sc = sd * cd, cc = cd * cd;
    R base = -(sc * __ldg(&A.duphi[i])) - cc * __ldg(&A.dvphi[i]) - ss * __ldg(&A.dulam[i]) - sc * __ldg(&A.dvlam[i]);
    if (A.variant == V_CART_DEEP_CUR || A.variant == V_SPHER_DEEP_CURR) return base;
    int ig = __ldg(&A.indep_g[i]);
    R tempc = __ldg(&A.v[i]) * __ldg(&A.ddphi[i]) + __ldg(&A.u[i]) * __ldg(&A.ddlam[i]);
    return (base * cgond(i + 1, m) + tempc * __ldg(&A.TSIHKD[(ig - 1) + A.NDEPTH * m])) *
           __ldg(&A.TFAK[(ig - 1) + A.NDEPTH * m]);
  }

  // Coefficients of point i (0-based), direction k, frequency m (0-based).
  __device__ Coefs<R> coef(int i, int k, int m) const {
    Coefs<R> c = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int KL = A.KL, ML = A.ML;
    const int kp = (k + 1 == KL) ? 0 : k + 1, km = (k == 0) ? KL - 1 : k - 1;
    const R sn = __ldg(&A.SINTH[k]), cs = __ldg(&A.COSTH[k]);
    const int IS = (sn >= R(0.)) ? 0 : 1, IT = 1 - IS, IC = (cs >= R(0.)) ? 0 : 1, ID = 1 - IC;
    const R z = R(0.);
    R tsi = 0;
    if (A.variant == V_CART_SHALLOW || A.variant == V_SPHER_SHALLOW || A.variant == V_CART_SHALLOW_CUR ||
        A.variant == V_SPHER_SHALLOW_CURR) {
      if (A.refr_d || A.variant == V_CART_SHALLOW_CUR || A.variant == V_SPHER_SHALLOW_CURR)
        tsi = __ldg(&A.TSIHKD[(__ldg(&A.indep_g[i]) - 1) + A.NDEPTH * m]);
    }
    switch (A.variant) {
      case V_CART_DEEP: {
        R dpn = dabs(cs * A.DELPH0 * __ldg(&A.GOM[m]));
        R sd = dabs(sn * __ldg(&A.GOM[m]));
        R dle = sd * __ldg(&A.della0[i]);
        c.sum = R(1.) - dle - dpn; c.lon1 = dle; c.lat11 = dpn;
      } break;
      case V_CART_SHALLOW: {
        R sd = dabs(sn), cd = dabs(cs * A.DELPH0), cg = cgond(i + 1, m), d0 = __ldg(&A.della0[i]);
        c.lon1 = sd * (cgond(klon(i, IS), m) + cg) * d0;
        c.lat11 = cd * (cgond(klat(i, IC, 0), m) + cg);
        c.sum = R(1.) - sd * (cgond(klon(i, IT), m) + cg) * d0 - cd * (cgond(klat(i, ID, 0), m) + cg);
        if (A.refr_d) {
          R t0 = thdd(i, k, m, tsi);
          R dtp = (t0 + thdd(i, kp, m, tsi)) * A.DELTHR, dtm = (t0 + thdd(i, km, m, tsi)) * A.DELTHR;
          c.sum = c.sum - dmax(z, dtp) + dmin(z, dtm);
          c.th1 = -dmin(z, dtp); c.th2 = dmax(z, dtm);
        }
      } break;
      case V_CART_DEEP_CUR:
      case V_SPHER_DEEP_CURR: {
        const bool sph = A.variant == V_SPHER_DEEP_CURR;
        R gom = __ldg(&A.GOM[m]);
        R cgs = gom * sn, cgc = gom * cs, d0 = __ldg(&A.della0[i]);
        auto wok1 = [&](int p) { return uv(A.u, p) + cgs; };
        auto wok2 = [&](int p) { return (uv(A.v, p) + cgc) * A.DELPH0; };
        R w1 = wok1(i + 1), w2 = wok2(i + 1);
        R dlw = (w1 + wok1(klon(i, 0))) * d0, dle = (w1 + wok1(klon(i, 1))) * d0;
        R dtc = R(1.) - dmax(z, dle) + dmin(z, dlw);
        c.lon2 = -dmin(z, dle); c.lon1 = dmax(z, dlw);
        if (!sph) {
          R dps = w2 + wok2(klat(i, 0, 0)), dpn = w2 + wok2(klat(i, 1, 0));
          dtc = dtc - dmax(z, dpn) + dmin(z, dps);
          c.lat21 = -dmin(z, dpn); c.lat11 = dmax(z, dps);
        } else if (A.reduced) {
          R wl1 = __ldg(&A.wlat[i]), wl2 = __ldg(&A.wlat[i + A.nsea]);
          R p1 = __ldg(&A.dpsn[i]), p2 = __ldg(&A.dpsn[i + A.nsea]);
          R dps = (w2 + wok2(klat(i, 0, 0)) * p1) * wl1, dps2 = (w2 + wok2(klat(i, 0, 1)) * p1) * (R(1.) - wl1);
          R dpn = (w2 + wok2(klat(i, 1, 0)) * p2) * wl2, dpn2 = (w2 + wok2(klat(i, 1, 1)) * p2) * (R(1.) - wl2);
          dtc = dtc - dmax(z, dpn) - dmax(z, dpn2) + dmin(z, dps) + dmin(z, dps2);
          c.lat21 = -dmin(z, dpn); c.lat22 = -dmin(z, dpn2); c.lat11 = dmax(z, dps); c.lat12 = dmax(z, dps2);
        } else {
          R dps = w2 + wok2(klat(i, 0, 0)) * __ldg(&A.dpsn[i]);
          R dpn = w2 + wok2(klat(i, 1, 0)) * __ldg(&A.dpsn[i + A.nsea]);
          dtc = dtc - dmax(z, dpn) + dmin(z, dps);
          c.lat11 = dmax(z, dps); c.lat21 = -dmin(z, dpn);
        }
        R t0 = thdd(i, k, ML - 1, tsi), tp = thdd(i, kp, ML - 1, tsi), tm = thdd(i, km, ML - 1, tsi);
        R dtp, dtm;
        if (sph) {
          R sp = A.DELTH0 * (sn + __ldg(&A.SINTH[kp])) * gom, sm = A.DELTH0 * (sn + __ldg(&A.SINTH[km])) * gom;
          R dr = __ldg(&A.drgm[i]);
          dtp = sp * dr + (t0 + tp) * A.DELTHR; dtm = sm * dr + (t0 + tm) * A.DELTHR;
        } else {
          dtp = (t0 + tp) * A.DELTHR; dtm = (t0 + tm) * A.DELTHR;
        }
        dtc = dtc - dmax(z, dtp) + dmin(z, dtm);
        c.th1 = -dmin(z, dtp); c.th2 = dmax(z, dtm);
        R dom = sidc(i, k, ML - 1) * A.DELFR0;
        c.sum = dtc - dabs(dom);
        c.sg1 = -dmin(z, dom) / R(1.1); c.sg2 = dmax(z, dom) * R(1.1);
      } break;
      case V_CART_SHALLOW_CUR:
      case V_SPHER_SHALLOW_CURR: {
        const bool sph = A.variant == V_SPHER_SHALLOW_CURR;
        const int mm = (m == 0) ? 0 : m - 1, mp = (m == ML - 1) ? ML - 1 : m + 1;
        R dfp = A.DELFR0 / __ldg(&A.FR[m]), dfm = A.DELFR0 / __ldg(&A.FR[mm]);
        R d0 = __ldg(&A.della0[i]);
        auto wok1 = [&](int p) { return uv(A.u, p) + sn * cgond(p, m); };
        auto wok2 = [&](int p) { return (uv(A.v, p) + cs * cgond(p, m)) * A.DELPH0; };
        R w1 = wok1(i + 1), w2 = wok2(i + 1);
        R dlw = (w1 + wok1(klon(i, 0))) * d0, dle = (w1 + wok1(klon(i, 1))) * d0;
        R dtc = R(1.) - dmax(z, dle) + dmin(z, dlw);
        c.lon1 = dmax(z, dlw); c.lon2 = -dmin(z, dle);
        if (!sph) {
          R dps = w2 + wok2(klat(i, 0, 0)), dpn = w2 + wok2(klat(i, 1, 0));
          dtc = dtc - dmax(z, dpn) + dmin(z, dps);
          c.lat11 = dmax(z, dps); c.lat21 = -dmin(z, dpn);
        } else if (A.reduced) {
          R wl1 = __ldg(&A.wlat[i]), wl2 = __ldg(&A.wlat[i + A.nsea]);
          R dps = w2 + __ldg(&A.dpsn[i]) * (wl1 * wok2(klat(i, 0, 0)) + (R(1.) - wl1) * wok2(klat(i, 0, 1)));
          R dps2 = dps * (R(1.) - wl1); dps = dps * wl1;
          R dpn = w2 + __ldg(&A.dpsn[i + A.nsea]) * (wl2 * wok2(klat(i, 1, 0)) + (R(1.) - wl2) * wok2(klat(i, 1, 1)));
          R dpn2 = dpn * (R(1.) - wl2); dpn = dpn * wl2;
          dtc = dtc - dmax(z, dpn) - dmax(z, dpn2) + dmin(z, dps) + dmin(z, dps2);
          c.lat11 = dmax(z, dps); c.lat12 = dmax(z, dps2); c.lat21 = -dmin(z, dpn); c.lat22 = -dmin(z, dpn2);
        } else {
          R dps = w2 + __ldg(&A.dpsn[i]) * wok2(klat(i, 0, 0));
          R dpn = w2 + __ldg(&A.dpsn[i + A.nsea]) * wok2(klat(i, 1, 0));
          dtc = dtc - dmax(z, dpn) + dmin(z, dps);
          c.lat11 = dmax(z, dps); c.lat21 = -dmin(z, dpn);
        }
        R t0 = thdd(i, k, m, tsi), tp = thdd(i, kp, m, tsi), tm = thdd(i, km, m, tsi);
        R dtp, dtm;
        if (sph) {
          R sp = A.DELTH0 * (sn + __ldg(&A.SINTH[kp])), sm = A.DELTH0 * (sn + __ldg(&A.SINTH[km]));
          R dr = __ldg(&A.drgm[i]), cg = cgond(i + 1, m);
          dtp = sp * dr * cg + (t0 + tp) * A.DELTHR; dtm = sm * dr * cg + (t0 + tm) * A.DELTHR;
        } else {
          dtp = (t0 + tp) * A.DELTHR; dtm = (t0 + tm) * A.DELTHR;
        }
        dtc = dtc - dmax(z, dtp) + dmin(z, dtm);
        c.th1 = -dmin(z, dtp); c.th2 = dmax(z, dtm);
        R s0 = sidc(i, k, m);
        R dop = (s0 + sidc(i, k, mp)) * dfp, dom = (s0 + sidc(i, k, mm)) * dfm;
        c.sg1 = -dmin(z, dop) / R(1.1); c.sg2 = dmax(z, dom) * R(1.1);
        c.sum = sph ? (dtc - dmax(z, dop) + dmin(z, dom)) : (dtc - dmax(z, dop) + dmin(z, dom));
      } break;
      case V_SPHER_DEEP: {
        R sda = dabs(sn), cda = dabs(cs * A.DELPH0);
        R sp = A.DELTH0 * (sn + __ldg(&A.SINTH[kp])), sm = A.DELTH0 * (sn + __ldg(&A.SINTH[km]));
        R gom = __ldg(&A.GOM[m]);
        R dpn = cda * (__ldg(&A.dpsn[i + A.nsea * IC]) + R(1.));
        R dle = sda * __ldg(&A.della0[i]);
        R dtc = cda * (__ldg(&A.dpsn[i + A.nsea * ID]) + R(1.)) + dle;
        R dr = __ldg(&A.drgm[i]);
        R dtp = dr * sp, dtm = dr * sm;
        dtc = dtc + dmax(z, dtp) - dmin(z, dtm);
        c.lat11 = gom * dpn; c.lon1 = gom * dle;
        c.th1 = -(gom * dmin(z, dtp)); c.th2 = gom * dmax(z, dtm);
        c.sum = R(1.) - gom * dtc;
        if (A.reduced) { R wl = __ldg(&A.wlat[i + A.nsea * IC]); c.lat12 = c.lat11 * (R(1.) - wl); c.lat11 = c.lat11 * wl; }
      } break;
      case V_SPHER_SHALLOW: {
        R sda = dabs(sn), cda = dabs(cs * A.DELPH0);
        R sp = A.DELTH0 * (sn + __ldg(&A.SINTH[kp])), sm = A.DELTH0 * (sn + __ldg(&A.SINTH[km]));
        R cg = cgond(i + 1, m), d0 = __ldg(&A.della0[i]);
        auto cgklat = [&](int ic) {
          R p = __ldg(&A.dpsn[i + A.nsea * ic]);
          if (A.reduced) {
            R wl = __ldg(&A.wlat[i + A.nsea * ic]);
            return cg + p * (wl * cgond(klat(i, ic, 0), m) + (R(1.) - wl) * cgond(klat(i, ic, 1), m));
          }
          return cg + p * cgond(klat(i, ic, 0), m);
        };
        R dtc = R(1.) - cda * cgklat(ID);
        c.lat11 = cda * cgklat(IC);
        dtc = dtc - sda * (cgond(klon(i, IT), m) + cg) * d0;
        c.lon1 = sda * (cgond(klon(i, IS), m) + cg) * d0;
        R dtp = __ldg(&A.drgm[i]) * cg, dtm;
        if (A.refr_d) {
          R t0 = thdd(i, k, m, tsi);
          dtm = dtp * sm + (t0 + thdd(i, km, m, tsi)) * A.DELTHR;
          dtp = dtp * sp + (t0 + thdd(i, kp, m, tsi)) * A.DELTHR;
        } else { dtm = dtp * sm; dtp = dtp * sp; }
        dtc = dtc - dmax(z, dtp) + dmin(z, dtm);
        c.th1 = -dmin(z, dtp); c.th2 = dmax(z, dtm);
        c.sum = dtc;
        if (A.reduced) { R wl = __ldg(&A.wlat[i + A.nsea * IC]); c.lat12 = c.lat11 * (R(1.) - wl); c.lat11 = c.lat11 * wl; }
      } break;
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
