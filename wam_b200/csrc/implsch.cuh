// IMPLSCH on sm_100a: one warp integrates one sea point.  A CTA stages the
// spectra of P consecutive sea points (32-byte sectors of the FL3(IJ,K,M)
// layout) into shared memory together with the static tables, and each warp
// then runs the reference's per-point statement sequence with its 32 lanes
// spread over directions, frequencies or spectral bins; spectral integrals
// and stresses are warp-shuffle reductions.
//
// Shared-memory rows of a point's spectrum use an odd stride ld >= KL, so
// lanes walking different frequencies of the same direction hit distinct
// banks.  The DIA runs quadruplet by quadruplet with lanes over directions:
// for fixed (MC,KH) the targets of different lanes within one target family
// are distinct (K1W..K21W are rotations) and the five frequency rows of a
// phase are distinct, so each of the two update phases is conflict-free and
// only the phases are separated by __syncwarp.
//
// Routine map (myWAveModel/WAM wam_source_module.f90 unless noted):
//   IMPLSCH :374-700        Src::run
//   SINPUT_ARD :2312-2738   sinput_ard        SINPUT_ST6 :4704-4925   sinput_st6
//   LFACTOR :4465-4700      sinput_st6        TAUWINDS :5555-5587     sinput_st6
//   SDISSIP_ARD :1704-1962  sdissip_ard       SDISSIP_ST6 :4929-5102  sdissip_st6
//   W3SWL6 :5106-5252       sdissip_st6       SNONLIN :2742-3047      snonlin
//   STRESSO :3164-3356      stresso_*         TAU_PHI_HF :3853-3966   tau_phi_hf
//   AIRSEA :868-971         airsea            W3FLX4 :5372-5443       w3flx4
//   WSIGSTAR :4250-4339     wsigstar          WAVNU2 :4343-4461       wavnu2
//   FRCUTINDEX :3569, FRCUTINDEX_ST6 :5447    IMPHFTAIL :3651-3731
//   SBOTTOM :1527-1589      WNFLUXES :3970-4054  (both in Src::run)
//   TOTAL_ENERGY/FEMEAN/WM1 wam_interface_module.f90:1342,207,1591
// Two reference computations whose results IMPLSCH never reads are not
// evaluated: TAU_WAVE_ATMOS (TAUNW of SINPUT_ST6) and, for ST6 without
// LCFLX, STRESSO (its TAUW is a dummy and PHIAW only feeds the flux module).
#pragma once
#include <cstdint>
#include <cfloat>
#include "wamgpu_config.hpp"
#include "spectral_tables.hpp"
#include "devmath.cuh"

namespace wamgpu {

// Shared-memory view of the small tables.
template <typename R> struct STabs {
  const R *FR, *DF, *DFIM, *DFIMOFR, *FR5, *FRM5, *RHOWG, *TH, *COSTH, *SINTH, *DELFL, *AF11, *RNL, *SATW, *WTAUHF,
      *SWELLFT, *SIG10, *DSII10;
  const int *K1W, *K2W, *K11W, *K21W, *INL, *IKP, *IKP1, *IKM, *IKM1, *INDSAT;
  __device__ void bind(const R* r, const int* i, const SmallLayout& L) {
    FR = r + L.FR; DF = r + L.DF; DFIM = r + L.DFIM; DFIMOFR = r + L.DFIMOFR; FR5 = r + L.FR5; FRM5 = r + L.FRM5;
    RHOWG = r + L.RHOWG_DFIM; TH = r + L.TH; COSTH = r + L.COSTH; SINTH = r + L.SINTH; DELFL = r + L.DELFL;
    AF11 = r + L.AF11; RNL = r + L.RNLCOEF; SATW = r + L.SATW; WTAUHF = r + L.WTAUHF; SWELLFT = r + L.SWELLFT;
    SIG10 = r + L.SIG10; DSII10 = r + L.DSII10;
    K1W = i + L.K1W; K2W = i + L.K2W; K11W = i + L.K11W; K21W = i + L.K21W; INL = i + L.INLCOEF;
    IKP = i + L.IKP; IKP1 = i + L.IKP1; IKM = i + L.IKM; IKM1 = i + L.IKM1; INDSAT = i + L.INDSAT;
  }
};

template <typename R> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

// Per-warp (per sea point) shared-memory workspace: bin (k,m) at k + ld*m.
// The source term SL and its diagonal derivative FL are always touched
// together, so they are interleaved (SF[b] = {SL, FL}): one 2-wide access per
// bin, which halves the load/store count of the DIA scatter.
template <typename R> struct WarpWS {
  using R2 = typename Vec2<R>::type;
  R2* SF;               // {SL, FL} per bin (first: 2*sizeof(R)-aligned)
  R *F, *SP;            // spectrum, positive input (SMIN when LCFLX)
  R* T;                 // 8 scratch rows of length scr (per frequency / direction; the DIA's buffer)
  uint8_t* LL;          // LLWS mask
  int ld, scr;
  __device__ R* t(int i) const { return T + i * scr; }
};

// Byte offset of the spectrum F inside a warp's workspace (after SF).
template <typename R> __host__ __device__ inline size_t ws_f_offset(int ld, int ML) { return 2 * (size_t)ld * ML * sizeof(R); }

template <typename R> __host__ __device__ inline size_t warp_ws_bytes(int ld, int ML, int need_sp, int scr) {
  size_t n = (size_t)ld * ML;
  size_t b = ((3 + (need_sp ? 1 : 0)) * n + 8 * (size_t)scr) * sizeof(R) + n + 16;  // + alignment of T
  return (b + 15) & ~size_t(15);
}

// Byte offset of the scratch rows T (16-byte aligned: the DIA keeps 2-wide
// values there).
template <typename R> __host__ __device__ inline size_t ws_t_offset(int ld, int ML, int need_sp) {
  size_t b = ws_f_offset<R>(ld, ML) + (size_t)ld * ML * sizeof(R) * (need_sp ? 2 : 1);
  return (b + 15) & ~size_t(15);
}

// WAVNU2 (:4343-4461) for one frequency: wavenumber and group velocity at
// angular frequency w0 and depth H by Newton's method.
// The hyperbolic functions are correctly rounded and nothing is contracted,
// so WN and CG equal the oracle's bit for bit; they are formed once per
// depth, outside the step.
template <typename R> __device__ __forceinline__ void wavnu2_one(R w0, R H, R& wn, R& cgv) {
  using P_ = Phys<R>;
  const R eps = R(1E-7);
  R k = (w0 < dsqrt(P_::G / H)) ? w0 / dsqrt(P_::G * H) : w0 * w0 / P_::G;
  R kold = 0;
  for (int i = 0; i < 15; ++i) {
    R dif = dabs(k - kold), rdif = (k != R(0)) ? dif / k : R(0);
    if (dif < eps && rdif < eps) break;
    kold = k;
    const R kh = kold * H, th = crtanh(kh);
    R f1 = rsub(rmul(P_::G * kold, th), rmul(w0, w0));
    R ch = crcosh(kh);
    R fd = (kh > R(25)) ? P_::G * th : radd(rmul(P_::G, th), (P_::G * kold * H) / (ch * ch));
    k = kold - f1 / fd;
  }
  wn = k;
  cgv = (R(2) * k * H > R(25)) ? w0 / k * R(0.5)
                               : w0 / k * R(0.5) * (R(1) + (R(2) * k * H / crsinh(R(2) * k * H)));
}

// Bytes of the small tables staged at the start of a CTA's shared memory.
template <typename R> __host__ __device__ inline size_t tables_bytes(const SmallLayout& L) {
  size_t b = (size_t)L.nreal * sizeof(R) + (size_t)L.nint * sizeof(int);
  return (b + 15) & ~size_t(15);
}

// Per-point outputs of IMPLSCH beyond the spectrum.
template <typename R> struct PointState {
  R TAUW, USTAR, Z0;
  R flx[7];  // PHIOC, TAUOC_X, TAUOC_Y, PHIBOT, TAUBOT_X, TAUBOT_Y, PHIAW
  // integer decisions of the step: JU, MIJ of the first and of the last
  // FRCUTINDEX call, LFACTOR iterations (ST6; 0 without reduction, -1 ST4)
  int JU = 0, MIJ1 = 0, MIJ2 = 0, LFIT = -1;
};

// Slots of the LFACTOR record (Src::lfrec).
enum LfRec { LF_TX0 = 0, LF_TY0, LF_TAU0, LF_TTOT, LF_RTAU0, LF_RLAST, LF_NIT, LF_REDUCE, LF_TX, LF_TY, LFREC_N };

template <typename R> struct Src {
  using P_ = Phys<R>;
  const DevTables<R>& T;
  const STabs<R>& S;
  WarpWS<R>& w;
  const int lane, ij, INDEP;
  const R U10, UDIR, ROAIRN, WSTAR, DEPTH;
  const R* ENH;  // MAKE_SHALLOW_SNL factors of the launch's points (ISNONLIN != 0), else null
  const int enh_ld;
  // When set, SINPUT_ARD records the sheltering sums entering every
  // frequency: rows XST0, XST1, YST0, YST1 of length ML (the adjoint's tape).
  R* shl = nullptr;
  // ST6: this point's WN and CG rows formed once from the depth (WAVNU2), or null.
  const R* wncg = nullptr;
  // When set, SINPUT_ST6 records what the adjoint of LFACTOR needs (lane 0
  // writes LFREC_N values): the first stress sums, |tau|, tau_tot, tau_vis
  // before its cap, RTAU after the first error and at the last iteration, the
  // iteration count, the reduce flag and the final stress sums.
  R* lfrec = nullptr;
  // When set, the step copies its LLWS masks here: bin b of the first
  // SINPUT call's mask at dll[b * dll_ld], of the last one's at
  // dll[(NS + b) * dll_ld] (test diagnostics of the integer decisions).
  uint8_t* dll = nullptr;
  uint8_t* llcopy = nullptr;  // when set, SINPUT_ST6 also writes its LLWS mask here (same layout)
  size_t dll_ld = 0;
  // ST6 LFACTOR: when lfout is set, lane 0 stores the RTAU of the last
  // iteration (0 when LFACTOR does not iterate); when lfreplay is set, the
  // step takes that value instead of iterating and repeats only the last
  // round, which gives the same LFACT and stress sums (the adjoint's
  // recomputation from a checkpoint).
  R* lfout = nullptr;
  const R* lfreplay = nullptr;
  __device__ Src(const DevTables<R>& t, const STabs<R>& s, WarpWS<R>& ws, int l, int ij_, int indep, R u10, R udir,
                 R roairn, R wstar, R depth, const R* enh, int enh_ld_)
      : T(t), S(s), w(ws), lane(l), ij(ij_), INDEP(indep), U10(u10), UDIR(udir), ROAIRN(roairn), WSTAR(wstar), DEPTH(depth),
        ENH(enh), enh_ld(enh_ld_) {}

  __device__ int KL() const { return T.KL; }
  __device__ int ML() const { return T.ML; }
  __device__ R tfak(int m) const { return __ldg(&T.TFAK[(INDEP - 1) + T.NDEPTH * m]); }
  __device__ R tcgond(int m) const { return __ldg(&T.TCGOND[(INDEP - 1) + T.NDEPTH * m]); }
  using R2 = typename Vec2<R>::type;
  __device__ static R2 r2(R a, R b) { R2 v; v.x = a; v.y = b; return v; }

  // Lane-strided walk over the bins of frequencies [0, nm): bin b = lane + 32 i
  // is direction k = b mod KL of frequency m = b div KL; (m, k) advance by
  // (32 div KL, 32 mod KL) with one carry instead of a division per bin.
  template <class Fn> __device__ __forceinline__ void for_bins(int nm, Fn&& fn) const {
    const int kl = KL(), n = kl * nm, q = 32 / kl, r = 32 - q * kl;
    int m = lane / kl, k = lane - m * kl;
    for (int b = lane; b < n; b += 32) {
      fn(m, k);
      k += r; m += q;
      if (k >= kl) { k -= kl; ++m; }
    }
  }

  // Sums of up to four rows of n terms, each in index order on its own lane
  // (lane q sums rows[q] starting from init[q]), broadcast to every lane.
  // The reference sums its spectral integrals in frequency order, and these
  // sums decide the cut-off index, so they are not formed as tree reductions.
  template <int NQ> __device__ void ordered_sums(R* const (&rows)[NQ], const R (&init)[NQ], int n, R (&out)[NQ]) const {
    __syncwarp();
    R acc = R(0);
    const R* row = rows[0];
#pragma unroll
    for (int q = 0; q < NQ; ++q)
      if (lane == q) { acc = init[q]; row = rows[q]; }
    if (lane < NQ)
      for (int i = 0; i < n; ++i) acc = radd(acc, row[i]);
#pragma unroll
    for (int q = 0; q < NQ; ++q) out[q] = __shfl_sync(0xffffffffu, acc, q);
    __syncwarp();
  }

  // TOTAL_ENERGY + FEMEAN (+ WM1 for AKMEAN) of the spectrum, and the same
  // masked by the wind-sea mask LLWS, in one pass (interface:1342-1410,
  // 207-286, 1591-1716): EMEAN, FMEAN, AKMEAN when asked, EMEANWS, FMEANWS.
  // Each frequency's two direction sums run on one lane; the frequency sums
  // run in order, with the reference's operations, on four or five lanes at
  // once (scratch rows 3-7, free wherever the step calls this).
  __device__ void integrals(const uint8_t* mask, R& emean, R& fmean, R* akmean, R& emeanws, R& fmeanws) const {
    const int kl = KL(), ml = ML(), ld = w.ld;
    R tail = 0, tailw = 0;
    for (int m = lane; m < ml; m += 32) {
      R t = 0, tw = 0;
      const R* f = w.F + ld * m;
      const uint8_t* mk = mask + ld * m;
      for (int k = 0; k < kl; ++k) { const R v = f[k]; t = t + v; tw = tw + (mk[k] ? v : R(0)); }
      integral_rows(m, t, tw, akmean != nullptr, tail, tailw);
    }
    integral_sums(tail, tailw, emean, fmean, akmean, emeanws, fmeanws);
  }
  // The row terms of frequency m from its direction sums t (all bins) and tw
  // (bins of the mask); lane (ML-1) mod 32 keeps the last row's sums as tails.
  __device__ __forceinline__ void integral_rows(int m, R t, R tw, bool ak, R& tail, R& tailw) const {
    const R DEL2 = dsqrt(P_::G) / P_::ZPI;
    w.t(3)[m] = rmul(t, S.DFIM[m]);
    w.t(4)[m] = rmul(t, S.DFIMOFR[m]);
    w.t(5)[m] = rmul(tw, S.DFIM[m]);
    w.t(6)[m] = rmul(tw, S.DFIMOFR[m]);
    if (ak) w.t(7)[m] = T.shallow ? rmul(t / dsqrt(tfak(m)), S.DFIM[m]) : rmul(rmul(t, S.DFIMOFR[m]), DEL2);
    if (m == ML() - 1) { tail = t; tailw = tw; }
  }
  // The frequency sums of the row terms in order, and the integrals.
  __device__ void integral_sums(R tail, R tailw, R& emean, R& fmean, R* akmean, R& emeanws, R& fmeanws) const {
    const int ml = ML();
    const R DEL2 = dsqrt(P_::G) / P_::ZPI;
    R* TE = w.t(3); R* TF = w.t(4); R* TEW = w.t(5); R* TFW = w.t(6); R* TW = w.t(7);
    tail = __shfl_sync(0xffffffffu, tail, (ml - 1) & 31);
    tailw = __shfl_sync(0xffffffffu, tailw, (ml - 1) & 31);
    R* rows[5] = {TE, TF, TEW, TFW, TW};
    const R init[5] = {rmul(T.MO_TAIL, tail), rmul(T.MM1_TAIL, tail), rmul(T.MO_TAIL, tailw), rmul(T.MM1_TAIL, tailw),
                       rmul(rmul(T.MM1_TAIL, DEL2), tail)};
    R sum[5];
    if (akmean) ordered_sums<5>(rows, init, ml, sum);
    else {
      R* rows4[4] = {TE, TF, TEW, TFW};
      const R init4[4] = {init[0], init[1], init[2], init[3]};
      R sum4[4];
      ordered_sums<4>(rows4, init4, ml, sum4);
      for (int q = 0; q < 4; ++q) sum[q] = sum4[q];
      sum[4] = R(0);
    }
    emean = dmax(sum[0], R(1.0E-12));
    fmean = emean / dmax(sum[1], R(1.0E-12));
    emeanws = dmax(sum[2], R(1.0E-12));
    fmeanws = emeanws / dmax(sum[3], R(1.0E-12));
    if (akmean) {
      const R wm = sum[4];
      *akmean = (emean > R(1.0E-12)) ? (emean / wm) * (emean / wm) : R(1.);
    }
  }

  // AIRSEA: u* and z0 from U10 and the wave stress (15 Newton steps).
  __device__ void airsea(R TAUW, R& USTAR, R& Z0) const {
    const R EPS1 = R(0.00001);
    R xlogxl = dlog(P_::XNLEV), alphaog = T.ALPHA / P_::G, xkutop = P_::XKAPPA * U10;
    R ustold = U10 * dsqrt(R(8.0E-4) + R(8.0E-5) * U10);
    R tauold = dmax(ustold * ustold, TAUW + EPS1);
    USTAR = dsqrt(tauold);
    R ustm1 = R(1.0) / dmax(USTAR, R(1.0E-6));
    R z0ch = 0;
    for (int it = 0; it < 15; ++it) {
      R x = TAUW / tauold;
      z0ch = alphaog * tauold / dsqrt(dmax(R(1.0) - x, EPS1));
      R z0vis = P_::RNUAIRM * ustm1, z0tot = z0ch + z0vis;
      R xologz0 = R(1.0) / (xlogxl - dlog(z0tot));
      R f = USTAR - xkutop * xologz0;
      R zz = ustm1 * (z0ch * (R(2.0) - R(3.0) * x) / (R(1.0) - x) - z0vis) / z0tot;
      R delf = R(1.0) - xkutop * (xologz0 * xologz0) * zz;
      USTAR = USTAR - f / delf;
      R taunew = dmax(USTAR * USTAR, TAUW + EPS1);
      USTAR = dsqrt(taunew);
      if (taunew == tauold) break;
      ustm1 = R(1.0) / dmax(USTAR, R(1.0E-6));
      tauold = taunew;
    }
    Z0 = z0ch;
  }

  // (the drag law's sums are rounded separately: u* decides the ST6 cut-off)
  __device__ void w3flx4(R& UST, R& Z0) const {
    R cd;
    if (U10 >= R(50.33)) { UST = R(2.026) * dsqrt(T.CDFAC); cd = (UST / U10) * (UST / U10); }
    else {
      cd = T.CDFAC * rsub(radd(R(8.058), rmul(R(0.967), U10)), rmul(R(0.016), U10 * U10)) * R(1E-4);
      UST = U10 * dsqrt(cd);
    }
    Z0 = P_::XNLEV * dexp(-R(0.4) / dsqrt(cd));
  }

  __device__ R wsigstar(R ustar, R z0) const {
    const R C1 = R(1.03E-3), C2 = R(0.04E-3), P1 = R(1.48), P2 = R(-0.21);
    R u = ustar * (R(1.0) / P_::XKAPPA) * (dlog(R(10.0)) - dlog(z0));
    u = dmax(u, R(1.0));
    R um1 = R(1.0) / u, c2u = C2 * dpow(u, P1), up2 = dpow(u, P2);
    R cdv = (C1 + c2u) * up2;
    R dcd = (P2 * C1 + (P1 + P2) * c2u) * up2 * um1;
    R sconv = R(1.0) + R(0.5) * u / cdv * dcd;
    return dmin(R(0.1), sconv * um1 * dpow(R(0.5) * P_::XKAPPA * (WSTAR * WSTAR * WSTAR), R(1.0) / R(3.0)));
  }

  // SINPUT_ARD: writes SL, FL, LL (and SP when kept) plus the per-frequency
  // sums of SPOS, SPOS*SIN, SPOS*COS that STRESSO integrates (scratch 0..2).
  // Sequential over frequency because of sheltering.
  // TAB = false is the reference's statement order (the forward step).  TAB =
  // true is the form the adjoint recomputes and linearises: the stress
  // direction's cosine and sine come from the stress components, COS(TH(K) -
  // USDIRP) from the direction tables, and (TPX^2+TPY^2)^(1/4) from two square
  // roots; it agrees with the reference form to a few ulp.
  template <bool TAB = false> __device__ void sinput_ard(R USTAR, R Z0) const {
    const int kl = KL(), ml = ML(), ld = w.ld;
    const R SWELLF = R(0.66), FU = R(0.022), FUD = R(-0.018), SWELLF4 = R(1.5E05), SWELLF5 = R(1.2), SWELLF7 = R(3.6E05);
    const R rog = P_::ROWATER * P_::G;
    const R const1 = T.BETAMAX / (P_::XKAPPA * P_::XKAPPA) / P_::ROWATER;
    const R nu = P_::RNUAIR;
    const R delabm1 = R(200) / (R(8.0) - R(0.3));
    const R shelter = dabs(T.TAUWSHELTER);
    R* ST = w.t(0); R* SX = w.t(1); R* SY = w.t(2);
    R sig_n = wsigstar(USTAR, Z0);
    R uo = 0, ao = 0;
    for (int m = lane; m < ml; m += 32) {
      R t = 0;
      for (int k = 0; k < kl; ++k) t = t + w.F[k + ld * m];
      R sig = P_::ZPI * S.FR[m];
      uo = uo + S.DFIM[m] * (sig * sig) * t;
      ao = ao + S.DFIM[m] * t;
    }
    R tiny = sizeof(R) == 4 ? R(FLT_MIN) : R(DBL_MIN);
    R uorbt = R(2.0) * dsqrt(tiny + warp_sum(uo));
    R aorb = R(2.0) * dsqrt(tiny + warp_sum(ao));
    R re = (R(4.0) / nu) * uorbt * aorb;
    R z0noz = dmax(P_::RNUAIRM / dmax(USTAR, R(0.0001)), R(0.04) * dmin(R(0.0005), Z0));
    R xi = (dlog10(dmax(aorb / z0noz, R(3.0))) - R(0.3)) * delabm1;
    int ind = min(199, max(1, (int)xi));  // xi >= 4.6 for finite input; clamp keeps NaN input in bounds
    R deli1 = dmin(R(1.0), xi - R(ind));
    R fww = S.SWELLFT[ind - 1] * (R(1.0) - deli1) + S.SWELLFT[ind] * deli1;
    R temp2 = fww * uorbt;
    R smooth = R(0.5) * dtanh((re - SWELLF4) / SWELLF7);
    R pturb = R(0.5) + smooth, pvisc = R(0.5) - smooth;
    R usg[2] = {(USTAR * (R(1.0) + sig_n)) * (USTAR * (R(1.0) + sig_n)), (USTAR * (R(1.0) - sig_n)) * (USTAR * (R(1.0) - sig_n))};
    R su = dsin(UDIR), cu = dcos(UDIR);
    R taux[2] = {usg[0] * su, usg[1] * su}, tauy[2] = {usg[0] * cu, usg[1] * cu};
    R xst[2] = {0, 0}, yst[2] = {0, 0};
    R rogoroair = rog / dmax(ROAIRN, R(1.0)), roairn_pvisc = ROAIRN * pvisc;
    for (int m = 0; m < ml; ++m) {
      if (shl && lane == 0) { shl[m] = xst[0]; shl[ml + m] = xst[1]; shl[2 * ml + m] = yst[0]; shl[3 * ml + m] = yst[1]; }
      R sig = P_::ZPI * S.FR[m], sig2 = sig * sig;
      R xk, cm;
      if (T.shallow) { xk = tfak(m); cm = xk * (R(1.0) / sig); }
      else { cm = sig / P_::G; xk = sig2 / P_::G; }
      R ustp[2], usdirp[2], cu_[2], su_[2], ucn[2], ucnz[2];
      for (int g = 0; g < 2; ++g) {
        R tpx = taux[g] - shelter * xst[g], tpy = tauy[g] - shelter * yst[g];
        if constexpr (TAB) {
          const R qq = tpx * tpx + tpy * tpy;
          ustp[g] = dsqrt(dsqrt(qq));
          const R rn = qq > R(0) ? R(1) / dsqrt(qq) : R(0);
          cu_[g] = qq > R(0) ? tpy * rn : R(1);
          su_[g] = tpx * rn;
          usdirp[g] = R(0);
        } else {
          ustp[g] = dpow(tpx * tpx + tpy * tpy, R(0.25));
          usdirp[g] = datan2(tpx, tpy);
          cu_[g] = su_[g] = R(0);
        }
        ucn[g] = ustp[g] * cm;
        ucnz[g] = P_::XKAPPA / (ucn[g] + T.ZALP);
      }
      R constf = rogoroair * cm * S.DFIM[m];
      R zcn = dlog(xk * Z0);
      R cnsn = (sig * const1) * ROAIRN;
      R coef = -(SWELLF * R(16.) * sig2 / (P_::G * P_::ROWATER));
      R coef5 = -(SWELLF5 * R(2.) * dsqrt(R(2.) * nu * sig) / P_::ROWATER);
      R dstab1 = coef5 * roairn_pvisc * xk, tmp1 = coef * ROAIRN;
      R px[2] = {0, 0}, py[2] = {0, 0}, st = 0, sx = 0, sy = 0;
      for (int k = lane; k < kl; k += 32) {
        R f = w.F[k + ld * m];
        R slp[2], flp[2];
        uint8_t ll = 0;
        for (int g = 0; g < 2; ++g) {
          R c;
          if constexpr (TAB) c = S.COSTH[k] * cu_[g] + S.SINTH[k] * su_[g];
          else c = dcos(S.TH[k] - usdirp[g]);
          R ufac = 0;
          if (c > R(0.01)) {
            R x = c * ucn[g], zlog = zcn + (TAB ? ucnz[g] * (R(1) / c) : ucnz[g] / c);
            if (zlog < R(0.0)) { R z2x = zlog * zlog * x; ufac = dexp(zlog) * z2x * z2x; ll = 1; }
          }
          R dstab = dstab1 + pturb * (tmp1 * (temp2 + (FU + FUD * c) * ustp[g]));
          slp[g] = cnsn * ufac;
          flp[g] = slp[g] + dstab;
          slp[g] = slp[g] * f;
          px[g] = px[g] + slp[g] * (constf * S.SINTH[k]);
          py[g] = py[g] + slp[g] * (constf * S.COSTH[k]);
        }
        int b = k + ld * m;
        R spos = R(0.5) * (slp[0] + slp[1]);  // >= 0
        if (w.SP) w.SP[b] = spos;
        st = st + spos; sx = sx + spos * S.SINTH[k]; sy = sy + spos * S.COSTH[k];
        R fl = R(0.5) * (flp[0] + flp[1]);
        w.SF[b] = r2(fl * f, fl);
        w.LL[b] = ll;
      }
      for (int g = 0; g < 2; ++g) { xst[g] = xst[g] + warp_sum(px[g]); yst[g] = yst[g] + warp_sum(py[g]); }
      st = warp_sum(st); sx = warp_sum(sx); sy = warp_sum(sy);
      if (lane == 0) { ST[m] = st; SX[m] = sx; SY[m] = sy; }
    }
    __syncwarp();
  }

  __device__ void tau_phi_hf(int mij, R ustar, R z0, R& tauhf, R& phihf) const {
    const R gm1 = R(1.0) / P_::G;
    R omegac = P_::ZPI * S.FR[mij - 1];
    R tauw = ustar * ustar, ust = ustar;
    R xloggz0 = dlog(P_::G * z0);
    R omegacc = dmax(omegac, T.X0TAUHF * P_::G / ustar);
    R sqrtz0og = dsqrt(z0 * gm1), sqrtgz0 = R(1.0) / sqrtz0og;
    R zinf = dlog(omegacc * sqrtz0og);
    R delz = dmax((R(0.0) - zinf) / R(18), R(0.0));
    tauhf = 0; phihf = 0;
    for (int j = 0; j < 19; ++j) {
      R y = dexp(zinf + R(j) * delz);
      R cm1 = y * sqrtgz0 * gm1;
      R zlog = dmin(xloggz0 + R(2.0) * dlog(cm1) + P_::XKAPPA / (ust * cm1 + T.ZALP), R(0.0));
      R z2 = zlog * zlog;
      R fnc2 = dexp(zlog) * (z2 * z2) * tauw * S.WTAUHF[j] * delz;
      ust = dsqrt(tauw);
      tauhf = tauhf + fnc2;
      phihf = phihf + fnc2 / y;
    }
    phihf = sqrtz0og * phihf;
  }

  // STRESSO from per-lane partial sums of the resolved part plus the
  // high-frequency tail.
  __device__ void stresso_finish(R USTAR, R Z0, int mij, R pphi, R px, R py, R& TAUW, R& PHIAW) const {
    const int kl = KL(), ld = w.ld;
    const R gm1 = R(1.0) / P_::G;
    const R cst = T.DELTH * ((P_::ZPI * P_::ZPI) * (P_::ZPI * P_::ZPI)) * gm1;
    R t1 = 0, t2 = 0;
    for (int k = lane; k < kl; k += 32) {
      R cw = dmax(dcos(S.TH[k] - UDIR), R(0.));
      R f = w.F[k + ld * (mij - 1)];
      t2 = t2 + f * (cw * cw);
      t1 = t1 + f * (cw * cw * cw);
    }
    pphi = warp_sum(pphi); px = warp_sum(px); py = warp_sum(py); t1 = warp_sum(t1); t2 = warp_sum(t2);
    R tau1, phi1;
    tau_phi_hf(mij, USTAR, Z0, tau1, phi1);
    R tauhf = cst * S.FR5[mij - 1] * gm1 * t1 * tau1;
    R phihf = P_::ROAIR * cst * S.FR5[mij - 1] * t2 * phi1;
    PHIAW = pphi + phihf;
    R xs = px / P_::ROAIR + tauhf * dsin(UDIR);
    R ys = py / P_::ROAIR + tauhf * dcos(UDIR);
    R tw = dsqrt(xs * xs + ys * ys);
    tw = dmin(tw, USTAR * USTAR - R(0.00001));
    TAUW = dmax(tw, R(0.));
  }
  __device__ R rhowgdfth(int m, int mij) const {
    R rw = S.RHOWG[m];
    return (m == mij - 1 && mij != ML()) ? R(0.5) * rw : rw;
  }
  __device__ R cmw(int m) const {
    return T.shallow ? tfak(m) * (R(1.0) / (P_::ZPI * S.FR[m])) : (P_::ZPI * S.FR[m]) * (R(1.0) / P_::G);
  }
  // ST4: the per-frequency sums were formed by SINPUT_ARD (scratch 0..2)
  __device__ void stresso_sums(R USTAR, R Z0, int mij, R& TAUW, R& PHIAW) const {
    const R* ST = w.t(0); const R* SX = w.t(1); const R* SY = w.t(2);
    R pphi = 0, px = 0, py = 0;
    for (int m = lane; m < mij; m += 32) {
      R rw = rhowgdfth(m, mij), cmr = cmw(m) * rw;
      pphi = pphi + ST[m] * rw; px = px + SX[m] * cmr; py = py + SY[m] * cmr;
    }
    stresso_finish(USTAR, Z0, mij, pphi, px, py, TAUW, PHIAW);
  }
  // ST6 with LCFLX: sums over the stored positive input
  __device__ void stresso_sp(R USTAR, R Z0, int mij, R& TAUW, R& PHIAW) const {
    const int kl = KL(), ld = w.ld;
    R pphi = 0, px = 0, py = 0;
    for_bins(mij, [&](int m, int k) {
      R rw = rhowgdfth(m, mij), cmr = cmw(m) * rw;
      R sp = dmax(w.SP[k + ld * m], R(0.));
      pphi = pphi + sp * rw;
      px = px + (sp * S.SINTH[k]) * cmr;
      py = py + (sp * S.COSTH[k]) * cmr;
    });
    stresso_finish(USTAR, Z0, mij, pphi, px, py, TAUW, PHIAW);
  }

  // FRCUTINDEX with the logarithms correctly rounded and the sums of the
  // ST6 form rounded separately: equal inputs give the oracle's MIJ.
  __device__ int frcutindex(R fm, R fmws, R ustar) const {
    R fpmh = R(2.5) / S.FR[0];
    R fppm = R(3.0) * P_::G / (R(28.0) * P_::ZPI * S.FR[0]);
    R fpm4 = dmax(dmax(fmws, fm) * fpmh, fppm / dmax(ustar, R(1.0E-6)));
    int mij = (int)lround((double)(crlog10(fpm4) * T.INV_LOG_CO)) + 1;
    return min(max(1, mij), ML());
  }
  __device__ int frcutindex_st6(R fmean, R ustar) const {
    const int nk = ML();
    R fxfm = R(6.) * P_::ZPI, fxpm = R(4.0) * P_::G / R(28.);
    R signk = P_::ZPI * S.FR[nk - 1];
    R facti1 = R(1.) / crlog(P_::CO), facti2 = rsub(R(1.), rmul(crlog(P_::ZPI * S.FR[0]), facti1));
    R fhigh = dmax(fxfm * fmean, fxpm / ustar);
    int nkh = min(nk, (int)radd(facti2, rmul(facti1, crlog(dmax(R(1.E-7), fhigh)))));
    int nkh1 = min(nk, nkh + 1);
    fhigh = dmin(signk, fhigh);
    return max(2, min(nkh1, (int)radd(facti2, rmul(facti1, crlog(dmax(R(1.E-7), fhigh))))));
  }

  // IMPHFTAIL: diagnostic tail above MIJ.
  __device__ void imphftail(int mij) const {
    const int kl = KL(), ml = ML(), ld = w.ld;
    R* t = w.t(7);
    for (int m = mij - 1 + lane; m < ml; m += 32) {
      if (T.shallow) { R akm1 = R(1.) / tfak(m); t[m] = (akm1 * akm1 * akm1) / tcgond(m); }
      else t[m] = S.FRM5[m];
    }
    __syncwarp();
    const R base = t[mij - 1];
    __syncwarp();
    for (int m = mij + lane; m < ml; m += 32) t[m] = t[m] / base;  // ratio of row m to row mij-1
    __syncwarp();
    for_bins(ml - mij, [&](int dm, int k) {
      const int m = mij + dm;
      w.F[k + ld * m] = t[m] * w.F[k + ld * (mij - 1)];
    });
    __syncwarp();
  }

  // SDISSIP_ARD: saturation-based whitecapping (SSDSC3 = SSDSC5 = 0).
  //
  // Frequency by frequency, lane k forms the saturation of direction k.  With
  // KL > 32 the directions 32..KL-1 (NX of them) are done for a group of
  // 32/NX frequencies at once, one lane per (frequency of the group,
  // direction): their saturations before the group, their whitecapping after
  // it.  The lanes holding a frequency's extra directions add them to that
  // frequency's maximum.  The maximum is exact and every bin keeps its own
  // formula, so the results do not depend on the grouping.
  __device__ R sat_facsat(int m) const {
    const R sig = P_::ZPI * S.FR[m];
    if (T.shallow) { const R xk = tfak(m); return (xk * xk * xk) * (R(1.0) / P_::ZPI) * tcgond(m); }
    const R xk = sig * sig / P_::G;
    return (xk * xk * xk) * (R(0.5) * (R(1.0) / P_::ZPI)) * P_::G / sig;
  }
  // saturation window sum of bin (k, m), without FACSAT
  __device__ R sat_window(int k, int m) const {
    const int kl = KL(), nw = 2 * T.NSDSNTH + 1;
    const R* fm = w.F + w.ld * m;
    R acc = 0;
    for (int j = 0; j < nw; ++j) acc = acc + S.SATW[k + kl * j] * fm[S.INDSAT[k + kl * j] - 1];
    return acc;
  }
  __device__ void sdissip_ard() const {
    const int kl = KL(), ml = ML(), ld = w.ld;
    const R tmp03 = R(1.0) / R(9.0E-4), c6 = R(0.3), c6m1 = R(1.) - c6;
    const int nx = kl > 32 ? kl - 32 : 0, gsz = nx > 0 ? 32 / nx : ml;
    const int lg = nx > 0 ? lane / nx : 0, lx = nx > 0 ? lane - lg * nx : 0;
    auto whitecap = [&](int k, int m, R bth, R temp1, R ssdsc2_sig) {
      R dd = dmax(R(0.), bth * tmp03 - R(1.0));
      R d = ssdsc2_sig * (temp1 + c6m1 * (dd * dd));
      int b = k + ld * m;
      R2 v = w.SF[b];
      v.x = v.x + d * w.F[b];
      v.y = v.y + d;
      w.SF[b] = v;
    };
    for (int m0 = 0; m0 < ml; m0 += gsz) {
      const int ng = min(gsz, ml - m0);
      const bool lact = nx > 0 && lg < ng;
      R bthx = 0, temp1x = 0;  // this lane's extra direction: saturation, TEMP1 of its frequency
      if (lact) bthx = sat_window(32 + lx, m0 + lg) * sat_facsat(m0 + lg);
      for (int g = 0; g < ng; ++g) {
        const int m = m0 + g;
        const R sig = P_::ZPI * S.FR[m], facsat = sat_facsat(m);
        R bth = 0, bmax = 0;
        if (lane < kl) { bth = sat_window(lane, m) * facsat; bmax = dmax(bmax, bth); }
        if (lact && lg == g) bmax = dmax(bmax, bthx);
        bmax = warp_max(bmax);
        R d0 = dmax(R(0.), bmax * tmp03 - R(1.0));
        R temp1 = c6 * (d0 * d0);
        if (lg == g) temp1x = temp1;
        if (lane < kl) whitecap(lane, m, bth, temp1, R(-2.2E-5) * sig);
      }
      if (lact) whitecap(32 + lx, m0 + lg, bthx, temp1x, R(-2.2E-5) * (P_::ZPI * S.FR[m0 + lg]));
    }
    __syncwarp();
  }

  // SNONLIN (DIA) for ISNONLIN = 0 (depth scaling from AKMEAN) or the
  // MAKE_SHALLOW_SNL table.
  //
  // Gather form of the reference's scatter.  For each MC the lanes first
  // compute the interactions of their directions for both KH and leave
  // {AD, DELAM} and {AD, DELAP} in a per-warp buffer; then every lane updates
  // only its own direction column of the five target rows (MC, MM, MM1, MP,
  // MP1), collecting the contributions whose partner tables point at it.  The
  // partner tables K1W, K2W, K11W and K21W are rotations of the directions by
  // a constant (checked on the host), so each source index is the column
  // rotated back.  The target rows of one MC are distinct (checked on the
  // host), and no two lanes write the same column, so the only ordering
  // needed is around the buffer.
  //
  // With KL > 32 the directions 32..KL-1 (NX of them) would take a second,
  // mostly idle pass per MC.  They are done for a batch of T.dia_batch
  // consecutive MCs at once, one lane per (MC of the batch, direction):
  //   - before the batch, one pass forms their interactions for every MC of
  //     the batch into the batch slots;
  //   - each MC's pass copies its slot into the buffer and, once the buffer
  //     is complete, leaves in the slot the four KH-summed gathers that the
  //     columns 32..KL-1 need;
  //   - after the batch, one pass updates those columns of the five target
  //     rows, one row kind at a time.  The rows of one kind are distinct
  //     within a batch (strictly increasing in MC, checked on the host), and
  //     the kinds are separated by barriers, so no two lanes write one bin
  //     at once.
  // The columns 32..KL-1 thus add the contributions of a batch kind by kind
  // rather than MC by MC: a different FP association, like the gather form.
  struct DiaMc {
    const R* rc;
    R ftemp, ftail;
    int rIC, rIP, rIP1, rIM, rIM1;       // gathered rows (offsets)
    int rMC, rMM, rMM1, rMP, rMP1;       // target rows (offsets; row 0 where not written)
    bool wMC, wMM, wMM1, wMP, wMP1;      // which targets this MC writes
  };
  __device__ DiaMc dia_mc(int mc, R enhfr) const {
    DiaMc d;
    const int4* e = T.diamc + 3 * (mc - 1);
    const int4 a = __ldg(e), b = __ldg(e + 1), c = __ldg(e + 2);
    d.rIC = a.x; d.rIP = a.y; d.rIP1 = a.z; d.rIM = a.w; d.rIM1 = b.x;
    d.rMC = b.y; d.rMM = b.z; d.rMM1 = b.w; d.rMP = c.x; d.rMP1 = c.y;
    d.wMC = c.z & 1; d.wMM = c.z & 2; d.wMM1 = c.z & 4; d.wMP = c.z & 8; d.wMP1 = c.z & 16;
    d.rc = S.RNL + RNL_STRIDE * (mc - 1);
    d.ftail = (c.z & 32) ? R(1) : d.rc[0];
    d.ftemp = S.AF11[c.w];
    if (T.shallow) d.ftemp = d.ftemp * (T.isnonlin == 0 ? enhfr : __ldg(&ENH[ij + (size_t)enh_ld * (mc - 1)]));
    return d;
  }

  // WIDE: more than 8 directions beyond the first 32 (KL > 40), so a batch
  // slot has more entries than lanes.  The common shapes compile without that
  // code in the MC loop.
  __device__ void snonlin(R AKMEAN) const {
    if (KL() > 40) snonlin_t<true>(AKMEAN);
    else snonlin_t<false>(AKMEAN);
  }
  template <bool WIDE> __device__ void snonlin_t(R AKMEAN) const {
    const int kl = KL(), ld = w.ld;
    R enhfr = R(1);
    if (T.shallow && T.isnonlin == 0) {
      enhfr = dmax(R(0.75) * DEPTH * AKMEAN, R(.5));
      enhfr = R(1.) + (R(5.5) / enhfr) * (R(1.) - R(.833) * enhfr) * dexp(R(-1.25) * enhfr);
    }
    R2* SF = w.SF; const R* F = w.F;
    R2* XM = reinterpret_cast<R2*>(w.T);  // [kh*kl + k] = {AD, DELAM}
    R2* XP = XM + 2 * kl;                 // [kh*kl + k] = {AD, DELAP}
    R2* XB = XP + 2 * kl;                 // batch slots, 4*NX per MC of the batch
    // rotation offsets of the partner tables, per KH (warp-uniform)
    int o1[2], o2[2], o11[2], o21[2];
    for (int kh = 0; kh < 2; ++kh) {
      o1[kh] = S.K1W[kl * kh] - 1; o2[kh] = S.K2W[kl * kh] - 1;
      o11[kh] = S.K11W[kl * kh] - 1; o21[kh] = S.K21W[kl * kh] - 1;
    }
    auto rot = [kl](int k, int o) { const int t = k + o; return t >= kl ? t - kl : t; };
    // interactions of direction k at one MC, both KH: {AD, DELAM} to xm[kh*skh],
    // {AD, DELAP} to xp[kh*skh]; AD and DELAD summed over KH to adc, delc
    auto interact = [&](const DiaMc& d, int k, R2* xm, R2* xp, int skh, R& adc, R& delc) {
      const Quad<R> c0 = ld4(d.rc), c1 = ld4(d.rc + 4);  // slots of RNLCOEF 0-4, 13-15
      const R g1 = c0.b, g2 = c0.c, g3 = c0.d, g4 = c1.a, g5 = c1.b, g6 = c1.c, g7 = c1.d, g8 = d.rc[8];
      const R fij = F[k + d.rIC] * d.ftail;
      adc = R(0); delc = R(0);
      for (int kh = 0; kh < 2; ++kh) {
        const int a1 = rot(k, o1[kh]), a11 = rot(k, o11[kh]), a2 = rot(k, o2[kh]), a21 = rot(k, o21[kh]);
        R sap = g1 * F[a1 + d.rIP] + g2 * F[a11 + d.rIP] + g3 * F[a1 + d.rIP1] + g4 * F[a11 + d.rIP1];
        R sam = g5 * F[a2 + d.rIM] + g6 * F[a21 + d.rIM] + g7 * F[a2 + d.rIM1] + g8 * F[a21 + d.rIM1];
        R fad1 = fij * (sap + sam);
        R fad2 = fad1 - R(2.) * sap * sam;
        fad1 = fad1 + fad2;
        R fcen = d.ftemp * fij;
        const R ad = fad2 * fcen;
        adc = adc + ad;
        delc = delc + fad1 * d.ftemp;
        xm[skh * kh] = r2(ad, (fij - R(2.) * sap) * T.DAL2 * fcen);
        xp[skh * kh] = r2(ad, (fij - R(2.) * sam) * T.DAL1 * fcen);
      }
    };
    // the target-row updates of column j from the KH-summed gathers
    // {a, dl} and {b, dm} of the kind's two partner tables, with the kind's
    // four weights (RNLCOEF slots 12 MM, 16 MM1, 20 MP, 24 MP1)
    auto upd = [&](const DiaMc& d, int slot, R2& v, R a, R dl, R b, R dm) {
      const Quad<R> c = ld4(d.rc + slot);
      v.x = v.x + (a * c.a + b * c.b); v.y = v.y + (dl * c.c + dm * c.d);
    };

    const int kmain = kl < 32 ? kl : 32;          // directions of the per-MC pass (lane = k)
    const int nx = kl > 32 ? kl - 32 : 0;         // directions done per batch
    const int bsz = max(1, nx > 0 ? T.dia_batch : T.MLSTHG);
    // this lane's batch item (MC lb of the batch, direction 32 + lx), and its
    // slot entry i = lane < 4*NX (T.dslot): the copy target in the buffer,
    // and the two buffer entries whose sum the columns 32..KL-1 need.  With
    // NX > 8 the entries 32 and up are read from the table where used.
    const int lb = nx > 0 ? lane / nx : 0, lx = nx > 0 ? lane - lb * nx : 0;
    int cdst = 0, sa = 0, sb = 0;
    if (lane < 4 * nx) { const int4 e = __ldg(T.dslot + lane); cdst = e.x; sa = e.y; sb = e.z; }
    for (int mc0 = 1; mc0 <= T.MLSTHG; mc0 += bsz) {
      const int nb = min(bsz, T.MLSTHG - mc0 + 1);
      const bool lact = nx > 0 && lb < nb;
      R ladc = R(0), ldelc = R(0);
      if (nx > 0) {
        if (lact) {
          const DiaMc d = dia_mc(mc0 + lb, enhfr);
          R2* xs = XB + 4 * nx * lb + lx;
          interact(d, 32 + lx, xs, xs + 2 * nx, nx, ladc, ldelc);
        }
        __syncwarp();
      }
      for (int b = 0; b < nb; ++b) {
        const DiaMc d = dia_mc(mc0 + b, enhfr);
        // 1. interactions (both KH) of this lane's direction; the batch's
        // directions come from the slot
        R adc = R(0), delc = R(0);
        if (lane < kmain) interact(d, lane, XM + lane, XP + lane, kl, adc, delc);
        if (lane < 4 * nx) XM[cdst] = XB[4 * nx * b + lane];
        if (WIDE)
          for (int i = lane + 32; i < 4 * nx; i += 32) XM[__ldg(T.dslot + i).x] = XB[4 * nx * b + i];
        __syncwarp();
        // 2. this lane's column j of the five target rows
        if (lane < kmain) {
          const int j = lane;
          const R2 m2a = XM[rot(j, kl - o2[0])], m2b = XM[kl + rot(j, kl - o2[1])];
          const R2 m21a = XM[rot(j, kl - o21[0])], m21b = XM[kl + rot(j, kl - o21[1])];
          const R2 p1a = XP[rot(j, kl - o1[0])], p1b = XP[kl + rot(j, kl - o1[1])];
          const R2 p11a = XP[rot(j, kl - o11[0])], p11b = XP[kl + rot(j, kl - o11[1])];
          R2 vC = SF[j + d.rMC], vM = SF[j + d.rMM], vM1 = SF[j + d.rMM1], vP = SF[j + d.rMP], vP1 = SF[j + d.rMP1];
          const R a2 = m2a.x + m2b.x, d2 = m2a.y + m2b.y, a21 = m21a.x + m21b.x, d21 = m21a.y + m21b.y;
          const R a1 = p1a.x + p1b.x, d1 = p1a.y + p1b.y, a11 = p11a.x + p11b.x, d11 = p11a.y + p11b.y;
          if (d.wMC) { vC.x = vC.x - R(2.) * adc; vC.y = vC.y - R(2.) * delc; SF[j + d.rMC] = vC; }
          if (d.wMM) { upd(d, 12, vM, a2, d2, a21, d21); SF[j + d.rMM] = vM; }
          if (d.wMM1) { upd(d, 16, vM1, a2, d2, a21, d21); SF[j + d.rMM1] = vM1; }
          if (d.wMP) { upd(d, 20, vP, a1, d1, a11, d11); SF[j + d.rMP] = vP; }
          if (d.wMP1) { upd(d, 24, vP1, a1, d1, a11, d11); SF[j + d.rMP1] = vP1; }
        }
        if (lane < 4 * nx) {
          const R2 u = XM[sa], v = XM[sb];
          XB[4 * nx * b + lane] = r2(u.x + v.x, u.y + v.y);
        }
        if (WIDE)
          for (int i = lane + 32; i < 4 * nx; i += 32) {
            const int4 e = __ldg(T.dslot + i);
            const R2 u = XM[e.y], v = XM[e.z];
            XB[4 * nx * b + i] = r2(u.x + v.x, u.y + v.y);
          }
        __syncwarp();  // the next MC overwrites the buffer
      }
      if (nx > 0) {
        // 3. the columns 32..KL-1 of the batch's target rows, one kind at a time
        const int j = 32 + lx;
        DiaMc d;
        R2 s2, s21, s1, s11;
        if (lact) {
          d = dia_mc(mc0 + lb, enhfr);
          const R2* xs = XB + 4 * nx * lb + lx;
          s2 = xs[0]; s21 = xs[nx]; s1 = xs[2 * nx]; s11 = xs[3 * nx];
        }
        if (lact && d.wMC) { R2 v = SF[j + d.rMC]; v.x = v.x - R(2.) * ladc; v.y = v.y - R(2.) * ldelc; SF[j + d.rMC] = v; }
        __syncwarp();
        if (lact && d.wMM) { R2 v = SF[j + d.rMM]; upd(d, 12, v, s2.x, s2.y, s21.x, s21.y); SF[j + d.rMM] = v; }
        __syncwarp();
        if (lact && d.wMM1) { R2 v = SF[j + d.rMM1]; upd(d, 16, v, s2.x, s2.y, s21.x, s21.y); SF[j + d.rMM1] = v; }
        __syncwarp();
        if (lact && d.wMP) { R2 v = SF[j + d.rMP]; upd(d, 20, v, s1.x, s1.y, s11.x, s11.y); SF[j + d.rMP] = v; }
        __syncwarp();
        if (lact && d.wMP1) { R2 v = SF[j + d.rMP1]; upd(d, 24, v, s1.x, s1.y, s11.x, s11.y); SF[j + d.rMP1] = v; }
        __syncwarp();  // the next batch overwrites the slots
      }
    }
  }

  // ---- ST6 ----------------------------------------------------------------
  // WAVNU2: wave number and group velocity per frequency -> scratch 0, 1
  // The depth is fixed between preparations, so the rows are normally formed
  // once per point (launch_wavnu2) and only read here.
  __device__ void wavnu2() const {
    R* WN = w.t(0); R* CG = w.t(1);
    if (wncg) {
      for (int m = lane; m < ML(); m += 32) { WN[m] = wncg[m]; CG[m] = wncg[ML() + m]; }
    } else {
      for (int m = lane; m < ML(); m += 32) wavnu2_one(dabs(P_::ZPI * S.FR[m]), DEPTH, WN[m], CG[m]);
    }
    __syncwarp();
  }

  // SINPUT_ST6 with LFACTOR: writes SL, FL, LL (and SP when kept); TAUW out;
  // nit: the LFACTOR iterations run (0 when the stress needs no reduction).
  // The positive growth rate D1 and the negative-input term D2 of every bin
  // are formed once (kept in SL and FL until the final pass).
  //
  // LFACTOR ends its iteration on |ERR| < 1.54E-4 (:4647-4672), so a last-bit
  // difference in the stress sums can change its iteration count and with it
  // every high-frequency growth rate.  Everything that enters those sums
  // follows the reference's operations: A = F*CGG/(ZPI*SIG) and
  // SDENSIG = S*SIG/CGG with the reference's divisions, sums rounded
  // separately (no FMA contraction), the TAUWINDS sums (:5555-5587) and the
  // sum of the LFACT in order, and the exponentials and wind-direction
  // cosines correctly rounded.  Equal inputs then give the oracle's
  // iteration count unless a per-bin TANH differs by an ulp.
  __device__ void sinput_st6(R USTAR, R& TAUW, int& nit, R& tail, R& tailw, bool ak) const {
    const int kl = KL(), nk = ML(), nk10 = T.NK10, ld = w.ld;
    const R* WN = w.t(0); const R* CG = w.t(1);
    R* SQB = w.t(2); R* LF = w.t(3); R* SDX = w.t(4); R* SDY = w.t(5); R* CI10 = w.t(6);
    const R cu = crcos(UDIR), su = crsin(UDIR), uproxy = R(32.) * USTAR;
    const R raw = ROAIRN / P_::ROWATER;
    // directional narrowness and saturation per frequency; CI10 = k/sigma
    for (int m = lane; m < nk; m += 32) {
      R sig = P_::ZPI * S.FR[m];
      const R* fm = w.F + ld * m;
      R2* sfm = w.SF + ld * m;  // SF.x keeps F*CG/ZS per bin until the growth rates replace it
      const R zs = P_::ZPI * sig, cg = CG[m];
      const RecipDiv<R> qzs(zs);
      R s = 0, mx = 0;
      for (int k = 0; k < kl; ++k) {
        const R a = qzs(rmul(fm[k], cg));
        sfm[k].x = a;
        s = s + a; mx = (k == 0) ? a : dmax(mx, a);
      }
      R s2 = 0;
      if (mx < R(1.0E-34)) s2 = R(kl);
      else {
        const RecipDiv<R> qmx(mx);
        for (int k = 0; k < kl; ++k) s2 = s2 + qmx(sfm[k].x);
      }
      R adensig = s * sig * T.DELTH, anar = R(1.0) / (s2 * T.DELTH);
      SQB[m] = dsqrt(anar * adensig * (WN[m] * WN[m] * WN[m]));
      CI10[m] = WN[m] / sig;
    }
    __syncwarp();
    // growth rates per bin, D1 to SF.x and D2 to SF.y, and the directional
    // sums of the positive stress spectrum (LFACTOR :4580-4595) in one pass
    // over each frequency row.  Only one of W1 (proj > 0) and W2 (proj < 0) is
    // nonzero, and the other term is +0 whatever its tanh, so one tanh per bin
    // gives the same D1, D2.
    for (int m = lane; m < nk; m += 32) {
      const R sig = P_::ZPI * S.FR[m], sqb = SQB[m], uci = uproxy * CI10[m];
      R bx = 0, by = 0;
      R2* sfm = w.SF + ld * m;
      const RecipDiv<R> qcg(CG[m]);
      for (int k = 0; k < kl; ++k) {
        const R a = sfm[k].x;  // F*CG/ZS, from the first pass
        R proj = rsub(rmul(uci, radd(rmul(S.COSTH[k], cu), rmul(S.SINTH[k], su))), R(1.));
        R w1 = dmax(R(0.), proj); w1 = w1 * w1;
        R w2 = dmin(R(0.), proj); w2 = w2 * w2;
        const bool up = proj > R(0.);
        const R g = R(2.8) - (R(1.) + dtanh(rsub(rmul(R(10.) * sqb, up ? w1 : w2), R(11.))));
        const R d1 = up ? raw * sig * g * sqb * w1 : R(0.);
        const R d2 = up ? R(0.) : raw * sig * R(0.09) * g * sqb * w2;
        sfm[k] = r2(d1, d2);
        const R sd = qcg(rmul(rmul(d1, a), sig));
        bx = radd(bx, rmul(dmax(R(0.), sd), S.COSTH[k]));
        by = radd(by, rmul(dmax(R(0.), sd), S.SINTH[k]));
      }
      SDX[m] = bx * T.DELTH; SDY[m] = by * T.DELTH;
    }
    __syncwarp();
    // extension to 10 Hz with an f^-2 tail (point-independent axis in S.SIG10/S.DSII10)
    if (nk < nk10) {
      const R signk = S.SIG10[nk - 1];
      for (int i = nk + lane; i < nk10; i += 32) {
        R r = (signk / S.SIG10[i]) * (signk / S.SIG10[i]);
        SDX[i] = SDX[nk - 1] * r; SDY[i] = SDY[nk - 1] * r;
        CI10[i] = S.SIG10[i] * R(0.101978);
      }
    }
    __syncwarp();
    const R* DS10 = S.DSII10;
    // TAUWINDS: the terms of both components go to rows 2 (SQB, done with)
    // and 7, and lanes 0 and 1 sum them in order
    R* TX = w.t(2); R* TY = w.t(7);
    const R gro = P_::G * P_::ROWATER;
    auto tauwinds = [&](R& tx, R& ty) {
      R* rows[2] = {TX, TY};
      const R init[2] = {R(0), R(0)};
      R sum[2];
      ordered_sums<2>(rows, init, nk10, sum);
      tx = gro * sum[0]; ty = gro * sum[1];
    };
    // LFACTOR: shrink the high-frequency input until the total stress matches u*^2
    R tau_tot = USTAR * USTAR * ROAIRN;
    R tau_vis = dmax(R(0.0), radd(-rmul(R(5.0E-5), U10), R(1.1E-3))) * (U10 * U10) * ROAIRN;
    tau_vis = dmin(R(0.95) * tau_tot, tau_vis);
    R tvx = tau_vis * cu, tvy = tau_vis * su;
    for (int i = lane; i < nk10; i += 32) { TX[i] = SDX[i] * CI10[i] * DS10[i]; TY[i] = SDY[i] * CI10[i] * DS10[i]; }
    R tauwx, tauwy;
    tauwinds(tauwx, tauwy);
    auto total = [&]() {
      const R ax = radd(tvx, tauwx), ay = radd(tvy, tauwy);
      return dsqrt(radd(rmul(ax, ax), rmul(ay, ay)));
    };
    R tau = total();
    R err = (tau - tau_tot) / tau_tot;
    if (lfrec && lane == 0) {
      lfrec[LF_TX0] = tauwx; lfrec[LF_TY0] = tauwy; lfrec[LF_TAU0] = tau; lfrec[LF_TTOT] = tau_tot;
      lfrec[LF_RTAU0] = err / R(90.); lfrec[LF_RLAST] = R(0); lfrec[LF_NIT] = R(0);
    }
    for (int i = lane; i < nk; i += 32) LF[i] = R(1.0);
    nit = 0;
    if (tau > tau_tot) {
      bool over = false;
      R rtau = err / R(90.), drtau = R(2.0);
      int sgn = (err >= R(0)) ? 1 : -1;
      // this lane's points of the 10 Hz axis (i = lane + 32 q) stay in
      // registers over the iterations; LF is stored once, from the last one
      constexpr int NQ = (MAX_NK10 + 31) / 32;
      R qx[NQ], qy[NQ], qc[NQ], qd[NQ], qa[NQ], qf[NQ];
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const int i = lane + 32 * q;
        const bool in = i < nk10;
        qx[q] = in ? SDX[i] : R(0); qy[q] = in ? SDY[i] : R(0); qc[q] = in ? CI10[i] : R(0);
        qd[q] = in ? DS10[i] : R(0); qa[q] = rsub(R(1.0), rmul(uproxy, qc[q])); qf[q] = R(1.0);
      }
      // Terms before the first negative exponent factor keep LFACT = 1 in
      // every iteration (RTAU stays positive), so their in-order partial sums
      // are formed once and each iteration continues from them.
      int L = nk10;
#pragma unroll
      for (int q = NQ - 1; q >= 0; --q) {
        const unsigned neg = __ballot_sync(0xffffffffu, lane + 32 * q < nk10 && qa[q] < R(0));
        if (neg) L = 32 * q + __ffs(neg) - 1;
      }
      R prex, prey;
      {
        __syncwarp();
        R acc = R(0);
        const R* row = lane == 0 ? TX : TY;
        if (lane < 2)
          for (int i = 0; i < L; ++i) acc = radd(acc, row[i]);
        prex = __shfl_sync(0xffffffffu, acc, 0); prey = __shfl_sync(0xffffffffu, acc, 1);
        __syncwarp();
      }
      // LFACT of the 10 Hz axis at RTAU r and the stress sums (the replay of a
      // stored RTAU)
      auto round = [&](R r) {
        if (lfrec && lane == 0) lfrec[LF_RLAST] = r;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
          const int i = lane + 32 * q;
          if (i >= L && i < nk10) {
            const R lf = dmin(R(1.0), crexp(rmul(qa[q], r)));
            qf[q] = lf;
            TX[i] = (qx[q] * lf) * qc[q] * qd[q];
            TY[i] = (qy[q] * lf) * qc[q] * qd[q];
          }
        }
        __syncwarp();
        R acc = lane == 0 ? prex : prey;
        const R* row = lane == 0 ? TX : TY;
        if (lane < 2)
          for (int i = L; i < nk10; ++i) acc = radd(acc, row[i]);
        tauwx = gro * __shfl_sync(0xffffffffu, acc, 0); tauwy = gro * __shfl_sync(0xffffffffu, acc, 1);
        __syncwarp();
      };
      R rlast = rtau;
      // Two iterations per round: with the sums at RTAU r the round also forms
      // those at the two RTAU the next iteration can take (one per sign of
      // ERR, from the same state update); the second iteration of the round
      // then takes the one its sign selects.  Rows 3-6 (LF, SDX, SDY, CI10)
      // are free here: their values are in the q registers, and LF is
      // stored after the loop.
      R* UX = w.t(3); R* UY = w.t(4); R* DX = w.t(5); R* DY = w.t(6);
      auto next_r = [&](int s_, R r) -> R {
        const bool ov = over || (s_ != sgn);
        const R d = ov ? dmax(R(0.5) * (R(1.0) + drtau), R(1.00010)) : drtau;
        return (s_ > 0) ? r * d : r * (R(1) / d);
      };
      auto step_state = [&]() {
        tau = total();
        err = (tau - tau_tot) / tau_tot;
        int sold = sgn;
        sgn = (err >= R(0)) ? 1 : -1;
        if (sgn != sold) over = true;
        if (over) drtau = dmax(R(0.5) * (R(1.0) + drtau), R(1.00010));
        rtau = (sgn > 0) ? rtau * drtau : rtau * (R(1) / drtau);
      };
      while (!lfreplay && nit < 80) {
        const R rA = rtau, rU = next_r(1, rA), rD = next_r(-1, rA);
        R qfU[NQ], qfD[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
          const int i = lane + 32 * q;
          qfU[q] = qf[q]; qfD[q] = qf[q];
          if (i >= L && i < nk10) {
            const R la = dmin(R(1.0), crexp(rmul(qa[q], rA)));
            const R lu = dmin(R(1.0), crexp(rmul(qa[q], rU)));
            const R lb = dmin(R(1.0), crexp(rmul(qa[q], rD)));
            qf[q] = la; qfU[q] = lu; qfD[q] = lb;
            TX[i] = (qx[q] * la) * qc[q] * qd[q]; TY[i] = (qy[q] * la) * qc[q] * qd[q];
            UX[i] = (qx[q] * lu) * qc[q] * qd[q]; UY[i] = (qy[q] * lu) * qc[q] * qd[q];
            DX[i] = (qx[q] * lb) * qc[q] * qd[q]; DY[i] = (qy[q] * lb) * qc[q] * qd[q];
          }
        }
        __syncwarp();
        R acc = (lane & 1) ? prey : prex;
        const R* row = lane == 0 ? TX : lane == 1 ? TY : lane == 2 ? UX : lane == 3 ? UY : lane == 4 ? DX : DY;
        if (lane < 6)
          for (int i = L; i < nk10; ++i) acc = radd(acc, row[i]);
        R sm[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) sm[q] = __shfl_sync(0xffffffffu, acc, q);
        __syncwarp();
        // the iteration at rA
        nit = nit + 1;
        rlast = rA;
        if (lfrec && lane == 0) lfrec[LF_RLAST] = rA;
        tauwx = gro * sm[0]; tauwy = gro * sm[1];
        step_state();
        if (dabs(err) < R(1.54E-4) || nit >= 80) break;
        // the iteration at the RTAU its sign selected (rtau equals rU or rD)
        const bool up = sgn > 0;
        nit = nit + 1;
        rlast = rtau;
        if (lfrec && lane == 0) lfrec[LF_RLAST] = rtau;
#pragma unroll
        for (int q = 0; q < NQ; ++q) qf[q] = up ? qfU[q] : qfD[q];
        tauwx = gro * (up ? sm[2] : sm[4]); tauwy = gro * (up ? sm[3] : sm[5]);
        step_state();
        if (dabs(err) < R(1.54E-4)) break;
      }
      if (lfreplay) {
        rlast = *lfreplay;
        nit = 1;
        round(rlast);
      }
      if (lfout && lane == 0) *lfout = rlast;
#pragma unroll
      for (int q = 0; q < NQ; ++q)
        if (lane + 32 * q < nk) LF[lane + 32 * q] = qf[q];
    } else if (lfout && lane == 0) {
      *lfout = R(0);
    }
    __syncwarp();
    bool reduce;
    {
      R* rows[1] = {LF};
      const R init[1] = {R(0)};
      R sum[1];
      ordered_sums<1>(rows, init, nk, sum);
      reduce = sum[0] < R(nk);
    }
    TAUW = dsqrt(radd(rmul(tauwx, tauwx), rmul(tauwy, tauwy)));
    if (lfrec && lane == 0) {
      lfrec[LF_NIT] = R(nit); lfrec[LF_REDUCE] = reduce ? R(1) : R(0); lfrec[LF_TX] = tauwx; lfrec[LF_TY] = tauwy;
    }
    // The source terms and the wind-sea mask per frequency row, and with them
    // the row sums of the (unchanged) spectrum, all bins and the mask's, that
    // the spectral integrals after SINPUT take: their row terms replace LF
    // (row 3, read first) and fill rows 4-7.
    tail = R(0); tailw = R(0);
    for (int m = lane; m < nk; m += 32) {
      const R lfm = LF[m];
      R t = 0, tw = 0;
      for (int k = 0; k < kl; ++k) {
        const int p = k + ld * m;
        const R2 v = w.SF[p];
        R d = v.x;
        if (reduce) d = d * lfm;
        R dtot = d - v.y;
        R f = w.F[p];
        w.SF[p] = r2(dtot * f, dtot);
        if (w.SP) w.SP[p] = d * f;
        const bool ll = d * f > R(0);
        w.LL[p] = ll;
        if (llcopy) llcopy[p] = ll;
        t = t + f; tw = tw + (ll ? f : R(0));
      }
      integral_rows(m, t, tw, ak, tail, tailw);
    }
    __syncwarp();
  }

  // SDISSIP_ST6 (T1 + T2 breaking) followed by W3SWL6 (swell dissipation)
  __device__ void sdissip_st6() const {
    const int kl = KL(), nk = ML(), ld = w.ld;
    const R* WN = w.t(0); const R* CG = w.t(1);
    R* ADF = w.t(2); R* T12 = w.t(3);
    const R bnt = R(0.035) * R(0.035);
    const R xfac = (R(1.0) - R(1.0) / P_::CO) / (P_::CO - R(1.0) / P_::CO);
    // per frequency: T1 and the T2 increment, and W3SWL6's row sum, first
    // maximum and narrowness (one pass over the row for the two sums)
    R* BN = w.t(4); R* AB = w.t(5);
    R ps = 0, amax = -R(1);
    int imax = 0;
    for (int m = lane; m < nk; m += 32) {
      R et = (P_::ZPI * bnt) / (CG[m] * (WN[m] * WN[m] * WN[m]));
      const R sig = P_::ZPI * S.FR[m];
      const R* fm = w.F + ld * m;
      const R cgs = CG[m] / (P_::ZPI * sig);
      R s = 0, sa = 0, mx = 0;
      for (int k = 0; k < kl; ++k) {
        const R f = fm[k], a = f * cgs;
        s = s + f;
        sa = sa + a;
        mx = (k == 0) ? a : dmax(mx, a);
      }
      R nex = dmax(R(0.0), s * T.DELTH - et) / et;
      R nex4 = (nex * nex) * (nex * nex);
      T12[m] = R(4.75E-6) * S.FR[m] * nex4;  // T1
      R dfii = (m > 0 && m < nk - 1) ? S.DF[m] * xfac : S.DF[m];
      ADF[m] = nex4 * dfii;
      R s2 = 0;
      if (mx < R(1.0E-34)) s2 = R(kl);
      else { const R rmx = R(1.) / mx; for (int k = 0; k < kl; ++k) s2 = s2 + (fm[k] * cgs) * rmx; }
      R anar = R(1.0) / (s2 * T.DELTH);
      AB[m] = sa;
      BN[m] = anar * (sa * sig * T.DELTH) * (WN[m] * WN[m] * WN[m]);
      ps = ps + sa * (P_::ZPI * S.DFIM[m] * sig) / CG[m];
      if (sa > amax) { amax = sa; imax = m; }
    }
    __syncwarp();
    // T2 is a cumulative sum over frequency: inclusive warp scan in chunks of 32
    R carry = 0;
    for (int base = 0; base < nk; base += 32) {
      int m = base + lane;
      R v = (m < nk) ? ADF[m] : R(0);
      for (int o = 1; o < 32; o <<= 1) { R u = __shfl_up_sync(0xffffffffu, v, o); if (lane >= o) v = v + u; }
      v = v + carry;
      if (m < nk) T12[m] = R(-1.0) * (dmax(R(0.0), T12[m]) + dmax(R(0.0), R(7.00E-5) * v));
      carry = __shfl_sync(0xffffffffu, v, 31);
    }
    __syncwarp();
    // first maximum over frequency (MAXLOC)
    for (int o = 16; o > 0; o >>= 1) {
      R oa = __shfl_xor_sync(0xffffffffu, amax, o);
      int oi = __shfl_xor_sync(0xffffffffu, imax, o);
      if (oa > amax || (oa == amax && oi < imax)) { amax = oa; imax = oi; }
    }
    R b1 = R(0.0041) * (R(2.) * dsqrt(warp_sum(ps)) * WN[imax]);
    __syncwarp();
    for (int m = lane; m < nk; m += 32) {
      R sig = P_::ZPI * S.FR[m];
      AB[m] = (AB[m] > R(1.E-30)) ? -(R(2.) / R(3.) * b1 * sig * dsqrt(BN[m])) : R(0);
    }
    __syncwarp();
    for_bins(nk, [&](int m, int k) {
      const int p = k + ld * m;
      const R f = w.F[p];
      R2 v = w.SF[p];
      v.x = (v.x + T12[m] * f) + AB[m] * f;
      v.y = (v.y + T12[m]) + AB[m];
      w.SF[p] = v;
    });
    __syncwarp();
  }

  // ---- the whole IMPLSCH step for this point --------------------------------
  // Every warp of the CTA runs the step (a warp past the last sea point
  // repeats the last point), and the warps pass the phases together: the
  // step's code is much larger than the instruction cache, and warps in
  // different phases would keep evicting each other's code.
  __device__ static void phase() { __syncthreads(); }
  __device__ void run(PointState<R>& ps) const {
    const int kl = KL(), ml = ML(), ld = w.ld;
    R TAUW = ps.TAUW, USTAR, Z0;
    R emean, fmean, akmean = 0, emeanws, fmeanws, phiaw = 0;
    const int ju = min(300, max((int)lround((double)(U10 / T.DELU)), 1));
    ps.JU = ju;
    // the first spectral integrals come with the masked ones after SINPUT
    // (neither SINPUT nor AIRSEA / W3FLX4 reads them, and F is unchanged)
    if (T.iphys == 2) { wavnu2(); w3flx4(USTAR, Z0); }
    else airsea(TAUW, USTAR, Z0);
    if (T.iphys == 1) sinput_ard(USTAR, Z0);
    R tail6 = 0, tailw6 = 0;
    if (T.iphys == 2) sinput_st6(USTAR, TAUW, ps.LFIT, tail6, tailw6, T.shallow && T.isnonlin == 0);
    phase();
    if (dll) copy_mask(0);
    if (T.iphys == 2) integral_sums(tail6, tailw6, emean, fmean, (T.shallow && T.isnonlin == 0) ? &akmean : nullptr, emeanws, fmeanws);
    else integrals(w.LL, emean, fmean, (T.shallow && T.isnonlin == 0) ? &akmean : nullptr, emeanws, fmeanws);
    int mij = (T.iphys == 2) ? frcutindex_st6(fmean, USTAR) : frcutindex(fmean, fmeanws, USTAR);
    ps.MIJ1 = mij;
    if (T.iphys == 2) { w3flx4(USTAR, Z0); }
    else { stresso_sums(USTAR, Z0, mij, TAUW, phiaw); airsea(TAUW, USTAR, Z0); }
    imphftail(mij);
    if (T.iphys == 1) { sinput_ard(USTAR, Z0); phase(); }
    if (T.iphys == 1) stresso_sums(USTAR, Z0, mij, TAUW, phiaw);
    else if (T.lcflx) { R td; stresso_sp(USTAR, Z0, mij, td, phiaw); }
    if (T.lcflx) {  // SMIN = SL - SPOS, kept in SP from here on
      for_bins(ml, [&](int m, int k) { const int p = k + ld * m; w.SP[p] = w.SF[p].x - w.SP[p]; });
      __syncwarp();
    }
    if (T.iphys == 1) sdissip_ard();
    else sdissip_st6();
    phase();
    snonlin(akmean);
    phase();
    // SBOTTOM factor per frequency (scratch 6); SL_BOT = SBO*F is formed on the fly
    R* SBO = w.t(6);
    if (T.shallow) {
      const R cst = R(-2.0) * R(0.038) / P_::G;
      for (int m = lane; m < ml; m += 32) {
        R wav = tfak(m);
        SBO[m] = cst * wav / dsinh(dmin(R(2.) * DEPTH * wav, R(50.)));
      }
      __syncwarp();
    }
    if (T.lcflx) {  // WNFLUXES on SSOURCE = SL - SMIN and SL_BOT
      const R rog = P_::ROWATER * P_::G, scdfm = R(0.5) * T.DELTH * (R(1.) - R(1.) / P_::CO);
      R a[6] = {0, 0, 0, 0, 0, 0};
      for_bins(mij, [&](int m, int k) {
        const int p = k + ld * m;
        R cfm = (m < mij - 1) ? rog * S.DFIM[m] : rog * scdfm * S.FR[m];
        R cm = T.shallow ? tfak(m) / (P_::ZPI * S.FR[m]) : P_::ZPI * S.FR[m] / P_::G;
        R src = w.SF[p].x - w.SP[p];
        a[0] = a[0] + src * cfm;
        a[1] = a[1] + cm * src * cfm * S.SINTH[k];
        a[2] = a[2] + cm * src * cfm * S.COSTH[k];
        if (T.shallow) {
          R bot = SBO[m] * w.F[p];
          a[3] = a[3] + bot * cfm;
          a[4] = a[4] + cm * bot * cfm * S.SINTH[k];
          a[5] = a[5] + cm * bot * cfm * S.COSTH[k];
        }
      });
      for (int i = 0; i < 6; ++i) a[i] = warp_sum(a[i]);
      R tau = P_::ROAIR * USTAR * USTAR;
      ps.flx[0] = phiaw - a[0];
      ps.flx[1] = tau * dsin(UDIR) - a[1];
      ps.flx[2] = tau * dcos(UDIR) - a[2];
      ps.flx[3] = -a[3]; ps.flx[4] = -a[4]; ps.flx[5] = -a[5];
      ps.flx[6] = phiaw;
    }
    // implicit integration with the growth limiter and the minimum-energy floor
    const R delt = T.DELT, fmx = dmax(fmeanws, fmean);
    R* C2 = w.t(2); R* LIM = w.t(3); R* FMIN = w.t(4);  // cos^2 spreading, limiter, floor
    for (int k = lane; k < kl; k += 32) { R c = dmax(R(0.), dcos(S.TH[k] - UDIR)); C2[k] = c * c; }
    for (int m = lane; m < ml; m += 32) {
      LIM[m] = USTAR * S.DELFL[m] * fmx;
      FMIN[m] = __ldg(&T.FLMINFR[(ju - 1) + 300 * m]);
    }
    __syncwarp();
    // one frequency row per lane: the update of its bins and, with it, the
    // row sums of the updated spectrum (all bins and the mask's) that the
    // spectral integrals take; their row terms replace LIM, FMIN and SBO
    // (rows 3, 4 and 6, read first) and fill row 5
    {
      R tail = 0, tailw = 0;
      for (int m = lane; m < ml; m += 32) {
        const R lim = LIM[m], fmin = FMIN[m], sbo = T.shallow ? SBO[m] : R(0);
        R t = 0, tw = 0;
        for (int k = 0; k < kl; ++k) {
          const int p = k + ld * m;
          R f0 = w.F[p];
          const R2 v = w.SF[p];
          R sl = v.x, fl = v.y;
          if (T.shallow) { sl = sl + sbo * f0; fl = fl + sbo; }
          R t1 = fdiv(delt * sl, dmax(R(1.), R(1.) - delt * fl));  // divisor >= 1
          R t3 = dmin(dabs(t1), lim);
          R f = f0 + ((t1 >= R(0)) ? t3 : -t3);
          f = dmax(f, fmin * C2[k]);
          w.F[p] = f;
          t = t + f; tw = tw + (w.LL[p] ? f : R(0));
        }
        integral_rows(m, t, tw, false, tail, tailw);
      }
      __syncwarp();
      integral_sums(tail, tailw, emean, fmean, nullptr, emeanws, fmeanws);
    }
    mij = (T.iphys == 2) ? frcutindex_st6(fmean, USTAR) : frcutindex(fmean, fmeanws, USTAR);
    ps.MIJ2 = mij;
    if (dll) copy_mask(1);
    imphftail(mij);
    ps.TAUW = TAUW; ps.USTAR = USTAR; ps.Z0 = Z0;
  }

  // LLWS mask of this point to plane q of the diagnostics
  __device__ void copy_mask(int q) const {
    const int ns = KL() * ML();
    for_bins(ML(), [&](int m, int k) { dll[((size_t)q * ns + k + KL() * m) * dll_ld] = w.LL[k + w.ld * m]; });
  }
};

}  // namespace wamgpu
