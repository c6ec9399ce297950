// Adjoint of IMPLSCH (ST4), one sea point per warp with the point's work
// arrays in shared memory.
//
// The forward pass is recomputed inside the step with the forward kernel's own
// lane-parallel routines (Src; SINPUT_ARD in its tabled-direction form, which
// the reverse sweep linearises), recording what the reverse sweep needs: the
// cut-off indices, AIRSEA's outputs, SINPUT's sheltering sums and SPOS sums per
// frequency, the first wind-sea mask and the source terms SL/FL.  The reverse
// sweep then runs the routines backwards with the lanes spread over the
// directions of a frequency (or over all bins where the step is elementwise):
// IMPHFTAIL, the implicit update, the DIA, SDISSIP_ARD, STRESSO and
// SINPUT_ARD (second call on F1, then the first call on F0), the spectral
// integrals and AIRSEA.  Scalar routines of one point (AIRSEA, TAU_PHI_HF,
// WSIGSTAR) are differentiated by two dual-number passes, one per half-warp.
// The statements follow the point-per-thread restatement in adjoint.cuh,
// which is the same linearisation.
//
// Shared memory of one warp: the forward workspace (SF = {SL, FL} per bin,
// F, 8 scratch rows, LL), then LAM (adjoint of the spectrum), 14 tape rows of
// ML values and the first LLWS mask.  After the update's adjoint SF holds
// {lambda_SL, lambda_FL}.  F holds F0, then F1 from the first IMPHFTAIL on;
// once the reverse sweep is done with F1 it is reloaded with F0 from global
// memory.
#pragma once
#include "adjoint.cuh"
#include "implsch.cuh"

namespace wamgpu {

template <typename R> __host__ __device__ inline size_t adjw_lam_offset(int ld, int ML, int scr) {
  return warp_ws_bytes<R>(ld, ML, 0, scr);
}
template <typename R> __host__ __device__ inline size_t adjw_at_offset(int ld, int ML, int scr) {
  size_t b = adjw_lam_offset<R>(ld, ML, scr) + (size_t)ld * ML * sizeof(R);
  return (b + 15) & ~size_t(15);
}
template <typename R> __host__ __device__ inline size_t adjw_ll1_offset(int ld, int ML, int scr) {
  return adjw_at_offset<R>(ld, ML, scr) + ((14 * (size_t)ML * sizeof(R) + 15) & ~size_t(15));
}
template <typename R> __host__ __device__ inline size_t adjw_ws_bytes(int ld, int ML, int scr) {
  return adjw_ll1_offset<R>(ld, ML, scr) + (((size_t)ld * ML + 15) & ~size_t(15));
}

template <typename R> struct AdjW {
  using P_ = Phys<R>;
  using R2 = typename Vec2<R>::type;
  Src<R>& s;
  const DevTables<R>& T;
  const STabs<R>& S;
  WarpWS<R>& w;
  const adj::ATabs<R>& A;
  const adj::PointIn<R>& P;
  const int lane;
  const R* F0g;     // the input spectrum in global memory (point ij, stride ldg)
  const size_t ldg;
  R *LAM, *AT;
  uint8_t* LL1;
  // recorded forward state
  int mij = 1, mij2 = 1, ju = 1;
  R us1 = 0, z01 = 0, tauw1 = 0, us2 = 0, z02 = 0, fmean = 0, fmeanws = 0, akmean = 0, fmx = 0;

  __device__ AdjW(Src<R>& src, const adj::ATabs<R>& a, const adj::PointIn<R>& p, const R* f0g, size_t ldg_, R* lam, R* at,
                  uint8_t* ll1)
      : s(src), T(src.T), S(src.S), w(src.w), A(a), P(p), lane(src.lane), F0g(f0g), ldg(ldg_), LAM(lam), AT(at),
        LL1(ll1) {}

  __device__ int KL() const { return T.KL; }
  __device__ int ML() const { return T.ML; }
  // tape rows: sheltering sums (q = 0,1 XST of the two gust branches, 2,3 YST), SX, SY per call; LSX, LSY
  __device__ R* shl_rows(int call) const { return AT + 4 * call * ML(); }
  __device__ R* sx_row(int call) const { return AT + (8 + 2 * call) * ML(); }
  __device__ R* sy_row(int call) const { return AT + (9 + 2 * call) * ML(); }
  __device__ R* lsx_row() const { return AT + 12 * ML(); }
  __device__ R* lsy_row() const { return AT + 13 * ML(); }
  __device__ static R2 r2(R a, R b) { R2 v; v.x = a; v.y = b; return v; }
  // end of a phase: every warp of the CTA runs the same sequence of phases
  __device__ static void phase() { __syncthreads(); }

  // ---- forward with recording --------------------------------------------------
  __device__ void forward(R TAUW0) {
    const int ml = ML(), ld = w.ld;
    ju = min(300, max((int)lround((double)(s.U10 / T.DELU)), 1));
    R emean, emeanws;
    akmean = 0;
    const bool need_ak = T.shallow && T.isnonlin == 0;
    s.airsea(TAUW0, us1, z01);
    s.shl = shl_rows(0);
    s.template sinput_ard<true>(us1, z01);
    phase();
    s.for_bins(ml, [&](int m, int k) { LL1[k + ld * m] = w.LL[k + ld * m]; });
    for (int m = lane; m < ml; m += 32) { sx_row(0)[m] = w.t(1)[m]; sy_row(0)[m] = w.t(2)[m]; }
    __syncwarp();
    s.integrals(w.LL, emean, fmean, need_ak ? &akmean : nullptr, emeanws, fmeanws);
    mij = s.frcutindex(fmean, fmeanws, us1);
    R phiaw;
    s.stresso_sums(us1, z01, mij, tauw1, phiaw);
    s.airsea(tauw1, us2, z02);
    s.imphftail(mij);  // F = F1 from here on
    phase();
    s.shl = shl_rows(1);
    s.template sinput_ard<true>(us2, z02);
    s.shl = nullptr;
    phase();
    for (int m = lane; m < ml; m += 32) { sx_row(1)[m] = w.t(1)[m]; sy_row(1)[m] = w.t(2)[m]; }
    __syncwarp();
    s.sdissip_ard();
    phase();
    s.snonlin(akmean);
    phase();
    fmx = dmax(fmeanws, fmean);
    update_rows();
    mij2 = cutoff_after_update();
  }

  // cos^2 spreading (row 2), limiter (3), floor (4) and SBOTTOM factor (6) of the update
  __device__ void update_rows() const {
    const int kl = KL(), ml = ML();
    R *C2 = w.t(2), *LIM = w.t(3), *FMIN = w.t(4), *SBO = w.t(6);
    for (int k = lane; k < kl; k += 32) { const R c = dmax(R(0.), dcos(S.TH[k] - s.UDIR)); C2[k] = c * c; }
    const R cst = R(-2.0) * R(0.038) / P_::G;
    for (int m = lane; m < ml; m += 32) {
      LIM[m] = us2 * S.DELFL[m] * fmx;
      FMIN[m] = __ldg(&T.FLMINFR[(ju - 1) + 300 * m]);
      if (T.shallow) { const R wav = s.tfak(m); SBO[m] = cst * wav / dsinh(dmin(R(2.) * s.DEPTH * wav, R(50.))); }
    }
    __syncwarp();
  }

  // The update's output at bin (m, k), as the forward step forms it.
  __device__ R updated(int m, int k) const {
    const int p = k + w.ld * m;
    const R f0 = w.F[p];
    const R2 v = w.SF[p];
    R sl = v.x, fl = v.y;
    if (T.shallow) { sl = sl + w.t(6)[m] * f0; fl = fl + w.t(6)[m]; }
    const R t1 = fdiv(T.DELT * sl, dmax(R(1.), R(1.) - T.DELT * fl));
    const R t3 = dmin(dabs(t1), w.t(3)[m]);
    const R f = f0 + ((t1 >= R(0)) ? t3 : -t3);
    return dmax(f, w.t(4)[m] * w.t(2)[k]);
  }

  // MIJ of the updated spectrum: the integrals (unmasked and with the second
  // LLWS) of the update's output, formed without storing it, with the
  // frequency sums in order as the forward step forms them (scratch rows 0,
  // 1, 5 and 7; rows 2, 3, 4 and 6 hold the update's factors).
  __device__ int cutoff_after_update() const {
    const int kl = KL(), ml = ML(), ld = w.ld;
    R *TE = w.t(0), *TF = w.t(1), *TEW = w.t(5), *TFW = w.t(7);
    R tail = 0, tailw = 0;
    for (int m = lane; m < ml; m += 32) {
      R t = 0, tw = 0;
      const uint8_t* mk = w.LL + ld * m;
      for (int k = 0; k < kl; ++k) {
        const R f = updated(m, k);
        t = t + f;
        tw = tw + (mk[k] ? f : R(0));
      }
      TE[m] = rmul(t, S.DFIM[m]); TF[m] = rmul(t, S.DFIMOFR[m]);
      TEW[m] = rmul(tw, S.DFIM[m]); TFW[m] = rmul(tw, S.DFIMOFR[m]);
      if (m == ml - 1) { tail = t; tailw = tw; }
    }
    tail = __shfl_sync(0xffffffffu, tail, (ml - 1) & 31);
    tailw = __shfl_sync(0xffffffffu, tailw, (ml - 1) & 31);
    R* rows[4] = {TE, TF, TEW, TFW};
    const R init[4] = {rmul(T.MO_TAIL, tail), rmul(T.MM1_TAIL, tail), rmul(T.MO_TAIL, tailw), rmul(T.MM1_TAIL, tailw)};
    R sum[4];
    s.template ordered_sums<4>(rows, init, ml, sum);
    const R e = dmax(sum[0], R(1.0E-12)), fm = e / dmax(sum[1], R(1.0E-12));
    const R ew = dmax(sum[2], R(1.0E-12)), fmw = ew / dmax(sum[3], R(1.0E-12));
    return T.iphys == 2 ? s.frcutindex_st6(fm, us2) : s.frcutindex(fm, fmw, us2);
  }

  // ---- reverse sweep ---------------------------------------------------------------

  // Jacobians of the two-input scalar routines: the two dual-number passes run
  // on the two half-warps at once (their branch decisions follow the values,
  // which both passes share) and are exchanged.
  // du, dv: this lane's derivatives of the outputs (u, v) along input 0
  // (lanes < 16) or input 1 (lanes >= 16).
  __device__ adj::Jac2<R> jac_split(R du, R dv) const {
    adj::Jac2<R> J;
    const bool hi = lane >= 16;
    const R ou = __shfl_xor_sync(0xffffffffu, du, 16), ov = __shfl_xor_sync(0xffffffffu, dv, 16);
    J.d00 = hi ? ou : du; J.d10 = hi ? ov : dv;
    J.d01 = hi ? du : ou; J.d11 = hi ? dv : ov;
    return J;
  }
  // d(USTAR, Z0) / d(U10, TAUW) of AIRSEA
  __device__ adj::Jac2<R> airsea_jac(R U10, R TAUW) const {
    using D = adj::Dual<R>;
    const bool hi = lane >= 16;
    D us, z0;
    adj::airsea(A, D(U10, hi ? R(0) : R(1)), D(TAUW, hi ? R(1) : R(0)), us, z0);
    return jac_split(us.d, z0.d);
  }
  // d(TAUHF, PHIHF) / d(USTAR, Z0) of TAU_PHI_HF, and TAUHF itself
  __device__ adj::Jac2<R> tauphi_jac(int mj, R ustar, R z0, R& tauhf) const {
    using D = adj::Dual<R>;
    const bool hi = lane >= 16;
    D th, ph;
    adj::tau_phi_hf(A, mj, D(ustar, hi ? R(0) : R(1)), D(z0, hi ? R(1) : R(0)), th, ph);
    tauhf = th.v;
    return jac_split(th.d, ph.d);
  }
  // WSIGSTAR and its derivatives with respect to USTAR and Z0
  __device__ R wsig_grad(R ustar, R z0, R& dus, R& dz0) const {
    using D = adj::Dual<R>;
    const bool hi = lane >= 16;
    const D v = adj::wsigstar(P, D(ustar, hi ? R(0) : R(1)), D(z0, hi ? R(1) : R(0)));
    const R o = __shfl_xor_sync(0xffffffffu, v.d, 16);
    dus = hi ? o : v.d;
    dz0 = hi ? v.d : o;
    return v.v;
  }

  // IMPHFTAIL^T: rows m >= mij were copied from row mij-1 with a ratio.
  __device__ void imphftail_adj(int mj) const {
    const int kl = KL(), ml = ML(), ld = w.ld;
    R* t = w.t(7);
    for (int m = mj - 1 + lane; m < ml; m += 32) {
      if (T.shallow) { const R akm1 = R(1.) / s.tfak(m); t[m] = (akm1 * akm1 * akm1) / s.tcgond(m); }
      else t[m] = S.FRM5[m];
    }
    __syncwarp();
    const R base = t[mj - 1];
    for (int k = lane; k < kl; k += 32) {
      R acc = LAM[k + ld * (mj - 1)];
      for (int m = mj; m < ml; ++m) {
        acc = acc + (t[m] / base) * LAM[k + ld * m];
        LAM[k + ld * m] = R(0);
      }
      LAM[k + ld * (mj - 1)] = acc;
    }
    __syncwarp();
  }

  // The implicit update^T: LAM (output -> input spectrum) in place, SF
  // replaced by {lambda_SL, lambda_FL}; adds to the adjoints of USTAR and FMX.
  __device__ void update_adj(R& lus, R& lfmx) const {
    const int ld = w.ld;
    const R delt = T.DELT;
    const R *C2 = w.t(2), *LIM = w.t(3), *FMIN = w.t(4), *SBO = w.t(6);
    R aus = 0, afmx = 0;
    s.for_bins(ML(), [&](int m, int k) {
      const int p = k + ld * m;
      const R f0 = w.F[p];
      const R2 v = w.SF[p];
      R sl = v.x, fl = v.y;
      if (T.shallow) { sl = sl + SBO[m] * f0; fl = fl + SBO[m]; }
      const R den_raw = R(1.) - delt * fl, den = dmax(R(1.), den_raw);
      const R rden = fdiv(R(1.), den);  // den >= 1
      const R t1 = fdiv(delt * sl, den), at1 = dabs(t1), lim = LIM[m];
      const R t3 = dmin(at1, lim);
      const R f = f0 + ((t1 >= R(0)) ? t3 : -t3);
      const R lf = (f < FMIN[m] * C2[k]) ? R(0) : LAM[p];  // the floor holds when it is selected
      R lf0 = lf, lt1 = 0;
      const R lt3 = (t1 >= R(0)) ? lf : -lf;
      if (lim < at1) { aus = aus + lt3 * S.DELFL[m] * fmx; afmx = afmx + lt3 * us2 * S.DELFL[m]; }
      else lt1 = (t1 < R(0)) ? -lt3 : lt3;
      const R lsl = lt1 * delt * rden;
      const R lfl = (R(1.) < den_raw) ? lt1 * t1 * rden * delt : R(0);
      if (T.shallow) lf0 = lf0 + SBO[m] * lsl;
      LAM[p] = lf0;
      w.SF[p] = r2(lsl, lfl);
    });
    lus = lus + warp_sum(aus);
    lfmx = lfmx + warp_sum(afmx);
    __syncwarp();
  }

  // SNONLIN^T (DIA), the transpose of the forward gather: for each MC the
  // lanes first form, for their directions and both KH, the adjoints of the
  // interaction's centre value and of its two partner sums from the adjoints
  // of the nine targets, and leave the partner-sum adjoints in a per-warp
  // buffer; then every lane adds to its own direction column of the five
  // gathered rows (IC, IP, IP1, IM, IM1) what the interactions that read that
  // column owe it.  The partner tables are rotations (checked on the host), so
  // the interaction that read column j through a table is found by rotating j
  // back.  Returns the adjoint of AKMEAN (ISNONLIN = 0 in shallow water).
  //
  // With KL > 32 the directions 32..KL-1 are done for a batch of consecutive
  // MCs at once, as in the forward DIA: one pass forms their adjoints for
  // every MC of the batch into the batch slots; each MC's pass copies its
  // slot into the buffer and leaves there the four KH-summed partner adjoints
  // that the columns 32..KL-1 gather; one pass after the batch adds to those
  // columns of the five gathered rows, one row kind at a time.  The gathered
  // rows repeat at both ends of the frequency range (rows clamped to 1 and
  // ML), so the host cuts the batches wherever one kind would add twice to a
  // row (T.dia_adj_starts).
  __device__ bool adj_batch_start(int mc) const {
    return mc > 128 || ((T.dia_adj_starts[(mc - 1) >> 6] >> ((mc - 1) & 63)) & 1ull);
  }
  // WIDE: KL > 40, as in the forward DIA.
  __device__ R snonlin_adj() const { return KL() > 40 ? snonlin_adj_t<true>() : snonlin_adj_t<false>(); }
  template <bool WIDE> __device__ R snonlin_adj_t() const {
    const int kl = KL(), ld = w.ld;
    const bool dyn = T.shallow && T.isnonlin == 0;
    R enhfr = R(1), denh = R(0);
    if (dyn) {
      const adj::Dual<R> e = adj::snl_enhfr(A, P, adj::Dual<R>(akmean, R(1)));
      enhfr = e.v; denh = e.d;
    }
    const R2* SF = w.SF;
    const R* F = w.F;
    R* XS = w.T;          // [kh*kl + k]: adjoint of SAP
    R* XM = XS + 2 * kl;  // adjoint of SAM
    R* XB = XM + 2 * kl;  // batch slots, 4*NX per MC of the batch
    int o1[2], o2[2], o11[2], o21[2];
    for (int kh = 0; kh < 2; ++kh) {
      o1[kh] = S.K1W[kl * kh] - 1; o2[kh] = S.K2W[kl * kh] - 1;
      o11[kh] = S.K11W[kl * kh] - 1; o21[kh] = S.K21W[kl * kh] - 1;
    }
    auto rot = [kl](int k, int o) { const int t = k + o; return t >= kl ? t - kl : t; };
    R lenh = 0;
    // adjoints of direction k's interactions at one MC, both KH: SAP to
    // xs[kh*skh], SAM to xm[kh*skh]; FIJ's (times FTAIL) summed over KH
    // returned
    auto interact = [&](const typename Src<R>::DiaMc& d, int mc, int k, R* xs, R* xm, int skh) -> R {
      const Quad<R> c0 = ld4(d.rc), c1 = ld4(d.rc + 4);  // RNLCOEF slots (rnl_slot)
      const R g1 = c0.b, g2 = c0.c, g3 = c0.d, g4 = c1.a, g5 = c1.b, g6 = c1.c, g7 = c1.d, g8 = d.rc[8];
      const R ftemp = d.ftemp, ftail = d.ftail;
      const R fij = F[k + d.rIC] * ftail;
      const R2 vC = SF[k + d.rMC];
      R xf[2];
      for (int kh = 0; kh < 2; ++kh) {
        const int a1 = rot(k, o1[kh]), a11 = rot(k, o11[kh]), a2 = rot(k, o2[kh]), a21 = rot(k, o21[kh]);
        const R sap = g1 * F[a1 + d.rIP] + g2 * F[a11 + d.rIP] + g3 * F[a1 + d.rIP1] + g4 * F[a11 + d.rIP1];
        const R sam = g5 * F[a2 + d.rIM] + g6 * F[a21 + d.rIM] + g7 * F[a2 + d.rIM1] + g8 * F[a21 + d.rIM1];
        R lad = 0, ldelad = 0, ldelap = 0, ldelam = 0;
        if (d.wMC) { lad = lad - R(2.) * vC.x; ldelad = ldelad - R(2.) * vC.y; }
        // target weights per row kind: slots 12 MM, 16 MM1, 20 MP, 24 MP1
        if (d.wMM) {
          const R2 u = SF[a2 + d.rMM], u21 = SF[a21 + d.rMM];
          const Quad<R> c = ld4(d.rc + 12);
          lad = lad + (c.a * u.x + c.b * u21.x); ldelam = ldelam + (c.c * u.y + c.d * u21.y);
        }
        if (d.wMM1) {
          const R2 u = SF[a2 + d.rMM1], u21 = SF[a21 + d.rMM1];
          const Quad<R> c = ld4(d.rc + 16);
          lad = lad + (c.a * u.x + c.b * u21.x); ldelam = ldelam + (c.c * u.y + c.d * u21.y);
        }
        if (d.wMP) {
          const R2 u = SF[a1 + d.rMP], u11 = SF[a11 + d.rMP];
          const Quad<R> c = ld4(d.rc + 20);
          lad = lad + (c.a * u.x + c.b * u11.x); ldelap = ldelap + (c.c * u.y + c.d * u11.y);
        }
        if (d.wMP1) {
          const R2 u = SF[a1 + d.rMP1], u11 = SF[a11 + d.rMP1];
          const Quad<R> c = ld4(d.rc + 24);
          lad = lad + (c.a * u.x + c.b * u11.x); ldelap = ldelap + (c.c * u.y + c.d * u11.y);
        }
        // ad = (fij S - 2P) ftemp fij, delad = (2 fij S - 2P) ftemp,
        // delap = (fij - 2 sam) DAL1 ftemp fij, delam = (fij - 2 sap) DAL2 ftemp fij
        const R S2 = sap + sam, P2 = sap * sam;
        const R lfij = lad * ftemp * (R(2) * fij * S2 - R(2) * P2) + ldelad * R(2) * S2 * ftemp +
                       ldelap * T.DAL1 * ftemp * (R(2) * fij - R(2) * sam) +
                       ldelam * T.DAL2 * ftemp * (R(2) * fij - R(2) * sap);
        const R lsap = lad * ftemp * fij * (fij - R(2) * sam) + ldelad * (R(2) * fij - R(2) * sam) * ftemp -
                       ldelam * R(2) * T.DAL2 * ftemp * fij;
        const R lsam = lad * ftemp * fij * (fij - R(2) * sap) + ldelad * (R(2) * fij - R(2) * sap) * ftemp -
                       ldelap * R(2) * T.DAL1 * ftemp * fij;
        if (dyn) {
          const R lft = lad * (fij * S2 - R(2) * P2) * fij + ldelad * (R(2) * fij * S2 - R(2) * P2) +
                        ldelap * (fij - R(2) * sam) * T.DAL1 * fij + ldelam * (fij - R(2) * sap) * T.DAL2 * fij;
          lenh = lenh + lft * S.AF11[mc - T.MFRSTLW];
        }
        xf[kh] = lfij * ftail;
        xs[skh * kh] = lsap;
        xm[skh * kh] = lsam;
      }
      return xf[0] + xf[1];
    };

    const int kmain = kl < 32 ? kl : 32;  // directions of the per-MC pass (lane = k)
    const int nx = kl > 32 ? kl - 32 : 0;
    // this lane's batch item (MC lb of the batch, direction 32 + lx), and its
    // slot entry i = lane < 4*NX (the adjoint's part of T.dslot): the copy
    // target in the buffer, and the two buffer entries whose sum the columns
    // 32..KL-1 need.  With NX > 8 the entries 32 and up are read where used.
    const int lb = nx > 0 ? lane / nx : 0, lx = nx > 0 ? lane - lb * nx : 0;
    const int4* aslot = T.dslot + 4 * nx;
    int cdst = 0, sa = 0, sb = 0;
    if (lane < 4 * nx) { const int4 e = __ldg(aslot + lane); cdst = e.x; sa = e.y; sb = e.z; }
    for (int mc0 = 1, nb = 0; mc0 <= T.MLSTHG; mc0 += nb) {
      nb = 1;
      if (nx == 0) nb = T.MLSTHG;
      else while (mc0 + nb <= T.MLSTHG && !adj_batch_start(mc0 + nb)) ++nb;
      const bool lact = nx > 0 && lb < nb;
      R lxf = R(0);
      if (nx > 0) {
        if (lact) {
          const int mc = mc0 + lb;
          R* xs = XB + 4 * nx * lb + lx;
          lxf = interact(s.dia_mc(mc, enhfr), mc, 32 + lx, xs, xs + 2 * nx, nx);
        }
        __syncwarp();
      }
      for (int b = 0; b < nb; ++b) {
        const int mc = mc0 + b;
        const typename Src<R>::DiaMc d = s.dia_mc(mc, enhfr);
        // 1. per interaction (k, kh) of this lane: adjoints of FIJ, SAP, SAM;
        // the batch's directions come from the slot
        R xfc = R(0);
        if (lane < kmain) xfc = interact(d, mc, lane, XS + lane, XM + lane, kl);
        if (lane < 4 * nx) XS[cdst] = XB[4 * nx * b + lane];
        if (WIDE)
          for (int i = lane + 32; i < 4 * nx; i += 32) XS[__ldg(aslot + i).x] = XB[4 * nx * b + i];
        __syncwarp();
        // 2. this lane's column j of the five gathered rows
        if (lane < kmain) {
          const int j = lane;
          const Quad<R> c0 = ld4(d.rc), c1 = ld4(d.rc + 4);
          const R g8 = d.rc[8];
          const R sp1 = XS[rot(j, kl - o1[0])] + XS[kl + rot(j, kl - o1[1])];
          const R sp11 = XS[rot(j, kl - o11[0])] + XS[kl + rot(j, kl - o11[1])];
          const R sm2 = XM[rot(j, kl - o2[0])] + XM[kl + rot(j, kl - o2[1])];
          const R sm21 = XM[rot(j, kl - o21[0])] + XM[kl + rot(j, kl - o21[1])];
          LAM[j + d.rIC] = LAM[j + d.rIC] + xfc;
          LAM[j + d.rIP] = LAM[j + d.rIP] + (c0.b * sp1 + c0.c * sp11);
          LAM[j + d.rIP1] = LAM[j + d.rIP1] + (c0.d * sp1 + c1.a * sp11);
          LAM[j + d.rIM] = LAM[j + d.rIM] + (c1.b * sm2 + c1.c * sm21);
          LAM[j + d.rIM1] = LAM[j + d.rIM1] + (c1.d * sm2 + g8 * sm21);
        }
        if (lane < 4 * nx) XB[4 * nx * b + lane] = XS[sa] + XS[sb];
        if (WIDE)
          for (int i = lane + 32; i < 4 * nx; i += 32) {
            const int4 e = __ldg(aslot + i);
            XB[4 * nx * b + i] = XS[e.y] + XS[e.z];
          }
        __syncwarp();  // the next MC overwrites the buffer
      }
      if (nx > 0) {
        // 3. the columns 32..KL-1 of the batch's gathered rows, one kind at a time
        const int j = 32 + lx;
        int rIC = 0, rIP = 0, rIP1 = 0, rIM = 0, rIM1 = 0;
        R vP = 0, vP1 = 0, vM = 0, vM1 = 0;
        if (lact) {
          const typename Src<R>::DiaMc d = s.dia_mc(mc0 + lb, enhfr);
          const Quad<R> c0 = ld4(d.rc), c1 = ld4(d.rc + 4);
          const R g8 = d.rc[8];
          const R* xs = XB + 4 * nx * lb + lx;
          const R sp1 = xs[0], sp11 = xs[nx], sm2 = xs[2 * nx], sm21 = xs[3 * nx];
          rIC = d.rIC; rIP = d.rIP; rIP1 = d.rIP1; rIM = d.rIM; rIM1 = d.rIM1;
          vP = c0.b * sp1 + c0.c * sp11; vP1 = c0.d * sp1 + c1.a * sp11;
          vM = c1.b * sm2 + c1.c * sm21; vM1 = c1.d * sm2 + g8 * sm21;
        }
        if (lact) LAM[j + rIC] = LAM[j + rIC] + lxf;
        __syncwarp();
        if (lact) LAM[j + rIP] = LAM[j + rIP] + vP;
        __syncwarp();
        if (lact) LAM[j + rIP1] = LAM[j + rIP1] + vP1;
        __syncwarp();
        if (lact) LAM[j + rIM] = LAM[j + rIM] + vM;
        __syncwarp();
        if (lact) LAM[j + rIM1] = LAM[j + rIM1] + vM1;
        __syncwarp();  // the next batch overwrites the slots
      }
    }
    return warp_sum(lenh) * denh;
  }

  // SDISSIP_ARD^T.  The saturation window is a rotation of the directions
  // (INDICESSAT(K, J) = K + J - NSDSNTH modulo KL, checked on the host), so
  // the transposed window sum is gathered per column like the DIA.  With
  // KL > 32 the directions 32..KL-1 are grouped over frequencies as in the
  // forward: before a group, one lane per (frequency, extra direction) forms
  // what does not depend on the frequency's maximum; after it, their
  // whitecapping adjoint and transposed window sum.  Each frequency of the
  // group keeps its row of the window's adjoint sources (LB) for that.
  __device__ void sdissip_adj() const {
    const int kl = KL(), ml = ML(), nw = 2 * T.NSDSNTH + 1, ns = T.NSDSNTH, ld = w.ld;
    const R tmp03 = R(1.0) / R(9.0E-4), c6 = R(0.3), c6m1 = R(1.) - c6;
    const int nx = kl > 32 ? kl - 32 : 0;
    // a group holds at most as many frequencies as the scratch rows have LB
    // rows (8*scr reals), for every KL
    const int gcap = (8 * w.scr) / kl;
    const int gsz = min(nx > 0 ? 32 / nx : ml, gcap);
    const int lg = nx > 0 ? lane / nx : 0, lx = nx > 0 ? lane - lg * nx : 0;
    R* LBG = w.T;  // [g*kl + k]: LB of frequency m0 + g, g < gsz
    auto window = [&](int k, const R* fm) {
      R acc = 0;
      int src = k - ns;
      src = src < 0 ? src + kl : src;
      for (int j = 0; j < nw; ++j) {
        acc = acc + S.SATW[k + kl * j] * fm[src];
        src = src + 1 == kl ? 0 : src + 1;
      }
      return acc;
    };
    auto window_t = [&](int c, const R* lbr) {
      R acc = 0;
      for (int j = 0; j < nw; ++j) {
        int k = c - j + ns;
        k = k < 0 ? k + kl : (k >= kl ? k - kl : k);
        acc = acc + S.SATW[k + kl * j] * lbr[k];
      }
      return acc;
    };
    for (int m0 = 0; m0 < ml; m0 += gsz) {
      const int ng = min(gsz, ml - m0);
      const bool lact = nx > 0 && lg < ng;
      // this lane's extra bin (32 + lx, m0 + lg): saturation, its share of
      // the TEMP1 adjoint and its own window source
      R bthx = 0, ltx = 0, lbx = 0, temp1x = 0;
      if (lact) {
        const int m = m0 + lg, b = 32 + lx + ld * m;
        const R ss = R(-2.2E-5) * (P_::ZPI * S.FR[m]);
        bthx = window(32 + lx, w.F + ld * m) * s.sat_facsat(m);
        const R2 v = w.SF[b];
        const R ldv = w.F[b] * v.x + v.y;
        ltx = ldv * ss;
        const R ddraw = bthx * tmp03 - R(1.0), dd = dmax(R(0.), ddraw);
        if (R(0.) < ddraw) lbx = ldv * ss * c6m1 * R(2) * dd * tmp03;
      }
      for (int g = 0; g < ng; ++g) {
        const int m = m0 + g;
        const R sig = P_::ZPI * S.FR[m], facsat = s.sat_facsat(m);
        const R* fm = w.F + ld * m;
        const bool own = lact && lg == g;
        R bth = 0, bmax = 0;
        int kmax = -1;
        if (lane < kl) {
          bth = window(lane, fm) * facsat;
          if (bmax < bth) { bmax = bth; kmax = lane; }
        }
        if (own && bmax < bthx) { bmax = bthx; kmax = 32 + lx; }
        // the first direction of largest saturation (none while all are <= 0)
        for (int o = 16; o > 0; o >>= 1) {
          const R ob = __shfl_xor_sync(0xffffffffu, bmax, o);
          const int ok = __shfl_xor_sync(0xffffffffu, kmax, o);
          if (bmax < ob || (ob == bmax && ok >= 0 && (kmax < 0 || ok < kmax))) { bmax = ob; kmax = ok; }
        }
        const R d0raw = bmax * tmp03 - R(1.0), d0 = dmax(R(0.), d0raw);
        const R temp1 = c6 * (d0 * d0), ssdsc2_sig = R(-2.2E-5) * sig;
        if (own) temp1x = temp1;
        R lt1 = 0, lb = 0;
        if (lane < kl) {
          const int b = lane + ld * m;
          const R ddraw = bth * tmp03 - R(1.0), dd = dmax(R(0.), ddraw);
          const R d = ssdsc2_sig * (temp1 + c6m1 * (dd * dd));
          const R2 v = w.SF[b];
          LAM[b] = LAM[b] + d * v.x;
          const R ldv = fm[lane] * v.x + v.y;
          lt1 = ldv * ssdsc2_sig;
          if (R(0.) < ddraw) lb = ldv * ssdsc2_sig * c6m1 * R(2) * dd * tmp03;
        }
        if (own) lt1 = lt1 + ltx;
        const R ltemp1 = warp_sum(lt1);
        const R lt1s = ltemp1 * c6 * R(2) * d0 * tmp03;
        R* LB = LBG + g * kl;
        if (lane < kl) LB[lane] = ((R(0.) < d0raw && lane == kmax) ? lb + lt1s : lb) * facsat;
        if (own) LB[32 + lx] = ((R(0.) < d0raw && 32 + lx == kmax) ? lbx + lt1s : lbx) * facsat;
        __syncwarp();
        if (lane < kl) LAM[lane + ld * m] = LAM[lane + ld * m] + window_t(lane, LB);
      }
      if (lact) {
        const int m = m0 + lg, c = 32 + lx, b = c + ld * m;
        const R ss = R(-2.2E-5) * (P_::ZPI * S.FR[m]);
        const R dd = dmax(R(0.), bthx * tmp03 - R(1.0));
        const R d = ss * (temp1x + c6m1 * (dd * dd));
        LAM[b] = LAM[b] + d * w.SF[b].x;
        LAM[b] = LAM[b] + window_t(c, LBG + lg * kl);
      }
      __syncwarp();  // the next group overwrites the LB rows
    }
  }

  // STRESSO^T for TAUW of SINPUT call `call` (spectrum Fs): to the adjoints of
  // its SPOS sums (rows LSX, LSY), of the cut-off row of the spectrum, of USTAR
  // and of Z0.
  __device__ void stresso_adj(int call, const R* Fs, R US, R Z0, R lTAU, R& lUS, R& lZ0) const {
    const int kl = KL(), ml = ML(), ld = w.ld;
    const R *SX = sx_row(call), *SY = sy_row(call);
    R px = 0, py = 0;
    for (int m = lane; m < mij; m += 32) {
      const R cmr = s.cmw(m) * s.rhowgdfth(m, mij);
      px = px + SX[m] * cmr;
      py = py + SY[m] * cmr;
    }
    px = warp_sum(px); py = warp_sum(py);
    const R gm1 = R(1.0) / P_::G;
    const R cst = T.DELTH * ((P_::ZPI * P_::ZPI) * (P_::ZPI * P_::ZPI)) * gm1;
    R t1 = 0;
    for (int k = lane; k < kl; k += 32) {
      const R cw = dmax(dcos(S.TH[k] - s.UDIR), R(0.));
      t1 = t1 + Fs[k + ld * (mij - 1)] * (cw * cw * cw);
    }
    t1 = warp_sum(t1);
    R tau1;
    const adj::Jac2<R> J = tauphi_jac(mij, US, Z0, tau1);
    const R kc = cst * S.FR5[mij - 1] * gm1;
    const R tauhf = kc * t1 * tau1;
    const R su = dsin(s.UDIR), cu = dcos(s.UDIR);
    const R xs = px / P_::ROAIR + tauhf * su, ys = py / P_::ROAIR + tauhf * cu;
    const R tw = dsqrt(xs * xs + ys * ys), cap = US * US - R(0.00001);
    const R twc = dmin(tw, cap);
    const R ltwc = (twc < R(0.)) ? R(0) : lTAU;
    R ltw = 0;
    if (cap < tw) lUS = lUS + ltwc * R(2) * US;
    else ltw = ltwc;
    const R lxs = tw > R(0) ? ltw * xs / tw : R(0), lys = tw > R(0) ? ltw * ys / tw : R(0);
    const R lpx = lxs / P_::ROAIR, lpy = lys / P_::ROAIR, ltauhf = lxs * su + lys * cu;
    const R lt1 = ltauhf * kc * tau1, ltau1 = ltauhf * kc * t1;
    for (int k = lane; k < kl; k += 32) {
      const R cw = dmax(dcos(S.TH[k] - s.UDIR), R(0.));
      LAM[k + ld * (mij - 1)] = LAM[k + ld * (mij - 1)] + lt1 * (cw * cw * cw);
    }
    lUS = lUS + ltau1 * J.d00;
    lZ0 = lZ0 + ltau1 * J.d01;
    R *LSX = lsx_row(), *LSY = lsy_row();
    for (int m = lane; m < ml; m += 32) {
      const R cmr = m < mij ? s.cmw(m) * s.rhowgdfth(m, mij) : R(0);
      LSX[m] = lpx * cmr;
      LSY[m] = lpy * cmr;
    }
    __syncwarp();
  }

  // SINPUT_ARD^T of call `call` on spectrum Fs.  lSF: adjoints of its SL/FL
  // outputs (null for the first call, whose SL/FL the step overwrites); rows
  // LSX/LSY: adjoints of its SPOS sums.  Adds to LAM and to the adjoints of
  // USTAR and Z0.
  __device__ void sinput_adj(int call, const R* Fs, R US, R Z0, const R2* lSF, R& lUS, R& lZ0) const {
    const int kl = KL(), ml = ML(), ld = w.ld;
    const R SWELLF = R(0.66), FU = R(0.022), FUD = R(-0.018), SWELLF4 = R(1.5E05), SWELLF5 = R(1.2), SWELLF7 = R(3.6E05);
    const R const1 = T.BETAMAX / (P_::XKAPPA * P_::XKAPPA) / P_::ROWATER;
    const R nu = P_::RNUAIR, rog = P_::ROWATER * P_::G;
    const R delabm1 = R(200) / (R(8.0) - R(0.3));
    const R shelter = dabs(T.TAUWSHELTER);
    const R ROAIRN = s.ROAIRN;
    // per-point prologue (recomputed); WSIGSTAR with its derivatives
    R dsig_us, dsig_z0;
    const R sig_n = wsig_grad(US, Z0, dsig_us, dsig_z0);
    R uo = 0, ao = 0;
    for (int m = lane; m < ml; m += 32) {
      R t = 0;
      for (int k = 0; k < kl; ++k) t = t + Fs[k + ld * m];
      const R sig = P_::ZPI * S.FR[m];
      uo = uo + S.DFIM[m] * (sig * sig) * t;
      ao = ao + S.DFIM[m] * t;
    }
    uo = warp_sum(uo); ao = warp_sum(ao);
    const R tiny = sizeof(R) == 4 ? R(FLT_MIN) : R(DBL_MIN);
    const R uorbt = R(2.0) * dsqrt(tiny + uo), aorb = R(2.0) * dsqrt(tiny + ao);
    const R re = (R(4.0) / nu) * uorbt * aorb;
    const R a1 = P_::RNUAIRM / dmax(US, R(0.0001)), a2 = R(0.04) * dmin(R(0.0005), Z0);
    const R z0noz = dmax(a1, a2);
    const R ratio = aorb / z0noz;
    const R xi = (dlog10(dmax(ratio, R(3.0))) - R(0.3)) * delabm1;
    const int ind = min(199, max(1, (int)xi));
    const R deli1 = dmin(R(1.0), xi - R(ind));
    const R fww = S.SWELLFT[ind - 1] * (R(1.0) - deli1) + S.SWELLFT[ind] * deli1;
    const R temp2 = fww * uorbt;
    const R zs = (re - SWELLF4) / SWELLF7, th = dtanh(zs);
    const R smooth = R(0.5) * th, pturb = R(0.5) + smooth, pvisc = R(0.5) - smooth;
    const R sgn[2] = {R(1), R(-1)};
    R usg[2];
    for (int g = 0; g < 2; ++g) { const R a = US * (R(1.0) + sgn[g] * sig_n); usg[g] = a * a; }
    const R su = dsin(s.UDIR), cu = dcos(s.UDIR);
    const R taux[2] = {usg[0] * su, usg[1] * su}, tauy[2] = {usg[0] * cu, usg[1] * cu};
    const R rogoroair = rog / dmax(ROAIRN, R(1.0));
    const R roairn_pvisc = ROAIRN * pvisc;
    const R* shl = shl_rows(call);
    const R *LSX = lsx_row(), *LSY = lsy_row();
    // reverse over frequency with the adjoints of the sheltering sums
    R lxst[2] = {0, 0}, lyst[2] = {0, 0}, ltaux[2] = {0, 0}, ltauy[2] = {0, 0};
    R lpvisc = 0, lpturb = 0, ltemp2 = 0;  // lpturb, ltemp2: this lane's part
    for (int m = ml - 1; m >= 0; --m) {
      const R xst[2] = {shl[m], shl[ml + m]}, yst[2] = {shl[2 * ml + m], shl[3 * ml + m]};
      const R sig = P_::ZPI * S.FR[m], sig2 = sig * sig;
      R xk, cm;
      if (T.shallow) { xk = s.tfak(m); cm = xk * (R(1.0) / sig); }
      else { cm = sig / P_::G; xk = sig2 / P_::G; }
      // cos and sin of the stress direction USDIRP = ATAN2(tpx, tpy) from the
      // stress components; cos(TH - USDIRP) and sin(TH - USDIRP) per bin then
      // follow from the direction tables
      R tpx[2], tpy[2], ustp[2], cu_[2], su_[2], ucn[2], ucnz[2];
      for (int g = 0; g < 2; ++g) {
        tpx[g] = taux[g] - shelter * xst[g]; tpy[g] = tauy[g] - shelter * yst[g];
        const R qq = tpx[g] * tpx[g] + tpy[g] * tpy[g];
        ustp[g] = dsqrt(dsqrt(qq));
        const R rn = qq > R(0) ? R(1) / dsqrt(qq) : R(0);
        cu_[g] = qq > R(0) ? tpy[g] * rn : R(1);
        su_[g] = tpx[g] * rn;
        ucn[g] = ustp[g] * cm;
        ucnz[g] = P_::XKAPPA / (ucn[g] + T.ZALP);
      }
      const R constf = rogoroair * cm * S.DFIM[m];
      const R zcn = dlog(xk * Z0);
      const R cnsn = (sig * const1) * ROAIRN;
      const R coef = -(SWELLF * R(16.) * sig2 / (P_::G * P_::ROWATER));
      const R coef5 = -(SWELLF5 * R(2.) * dsqrt(R(2.) * nu * sig) / P_::ROWATER);
      const R dstab1 = coef5 * roairn_pvisc * xk;
      const R tmp1 = coef * ROAIRN;
      const R lSX = LSX[m], lSY = LSY[m];
      R q[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // lustp[2], lusdirp[2], lucn[2], lucnz[2], lzcn, ldstab1
      for (int k = lane; k < kl; k += 32) {
        const int b = k + ld * m;
        const R f = Fs[b];
        const R sk = S.SINTH[k], ck = S.COSTH[k];
        R c[2], ufac[2], slpu[2], zlog[2], xx[2], ez[2], rc[2];
        bool act[2];
        for (int g = 0; g < 2; ++g) {
          c[g] = ck * cu_[g] + sk * su_[g];
          ufac[g] = 0; act[g] = false; zlog[g] = 0; xx[g] = 0; ez[g] = 0; rc[g] = 0;
          if (c[g] > R(0.01)) {
            rc[g] = R(1) / c[g];
            xx[g] = c[g] * ucn[g];
            zlog[g] = zcn + ucnz[g] * rc[g];
            if (zlog[g] < R(0.0)) {
              const R z2x = zlog[g] * zlog[g] * xx[g];
              ez[g] = dexp(zlog[g]);
              ufac[g] = ez[g] * z2x * z2x;
              act[g] = true;
            }
          }
          slpu[g] = cnsn * ufac[g];
        }
        const R dst0 = dstab1 + pturb * (tmp1 * (temp2 + (FU + FUD * c[0]) * ustp[0]));
        const R dst1 = dstab1 + pturb * (tmp1 * (temp2 + (FU + FUD * c[1]) * ustp[1]));
        const R fl = R(0.5) * ((slpu[0] + dst0) + (slpu[1] + dst1));
        R lsl = 0, lfl_out = 0;
        if (lSF) { const R2 v = lSF[b]; lsl = v.x; lfl_out = v.y; }
        const R lfl = lsl * f + lfl_out;
        R lf = lsl * fl;
        const R lspos = lSX * S.SINTH[k] + lSY * S.COSTH[k];
        for (int g = 0; g < 2; ++g) {
          const R lslpf = R(0.5) * lspos + lxst[g] * (constf * S.SINTH[k]) + lyst[g] * (constf * S.COSTH[k]);
          const R lflp = R(0.5) * lfl;
          const R lslpu = lflp + lslpf * f;
          lf = lf + lslpf * slpu[g];
          const R ldstab = lflp;
          const R lufac = lslpu * cnsn;
          q[9] = q[9] + ldstab;
          lpturb = lpturb + ldstab * (tmp1 * (temp2 + (FU + FUD * c[g]) * ustp[g]));
          ltemp2 = ltemp2 + ldstab * pturb * tmp1;
          R lc = ldstab * pturb * tmp1 * FUD * ustp[g];
          q[g] = q[g] + ldstab * pturb * tmp1 * (FU + FUD * c[g]);
          if (act[g]) {
            const R e = ez[g], z2x = zlog[g] * zlog[g] * xx[g];
            const R lzlog = lufac * e * z2x * (z2x + R(4) * zlog[g] * xx[g]);
            const R lx = lufac * e * R(2) * z2x * zlog[g] * zlog[g];
            lc = lc + lx * ucn[g];
            q[4 + g] = q[4 + g] + lx * c[g];
            q[8] = q[8] + lzlog;
            q[6 + g] = q[6 + g] + lzlog * rc[g];
            lc = lc - lzlog * ucnz[g] * (rc[g] * rc[g]);
          }
          q[2 + g] = q[2 + g] + lc * (sk * cu_[g] - ck * su_[g]);  // sin(TH - USDIRP)
        }
        LAM[b] = LAM[b] + lf;
      }
      for (int i = 0; i < 10; ++i) q[i] = warp_sum(q[i]);
      for (int g = 0; g < 2; ++g) {
        const R d = ucn[g] + T.ZALP;
        const R lucn = q[4 + g] - q[6 + g] * P_::XKAPPA / (d * d);
        const R lustp = q[g] + lucn * cm;
        const R qq = tpx[g] * tpx[g] + tpy[g] * tpy[g];
        R ltpx = 0, ltpy = 0;
        if (qq > R(0)) {
          const R lq = lustp * R(0.25) * (R(1) / (ustp[g] * ustp[g] * ustp[g]));  // d qq^(1/4) / d qq
          ltpx = lq * R(2) * tpx[g] + q[2 + g] * tpy[g] / qq;
          ltpy = lq * R(2) * tpy[g] - q[2 + g] * tpx[g] / qq;
        }
        ltaux[g] = ltaux[g] + ltpx;
        ltauy[g] = ltauy[g] + ltpy;
        lxst[g] = lxst[g] - shelter * ltpx;
        lyst[g] = lyst[g] - shelter * ltpy;
      }
      lZ0 = lZ0 + q[8] / Z0;
      lpvisc = lpvisc + q[9] * coef5 * ROAIRN * xk;
    }
    lpturb = warp_sum(lpturb);
    ltemp2 = warp_sum(ltemp2);
    // prologue^T
    R lsig_n = 0;
    for (int g = 0; g < 2; ++g) {
      const R lusg = ltaux[g] * su + ltauy[g] * cu;
      const R a = US * (R(1.0) + sgn[g] * sig_n);
      const R la = R(2) * a * lusg;
      lUS = lUS + la * (R(1.0) + sgn[g] * sig_n);
      lsig_n = lsig_n + la * US * sgn[g];
    }
    const R lsmooth = lpturb - lpvisc;
    const R lre = lsmooth * R(0.5) * (R(1) - th * th) / SWELLF7;
    R luorbt = ltemp2 * fww, laorb = 0;
    const R lfww = ltemp2 * uorbt;
    const R ldeli1 = lfww * (S.SWELLFT[ind] - S.SWELLFT[ind - 1]);
    const R lxi = ((xi - R(ind)) < R(1.0)) ? ldeli1 : R(0);
    R lz0noz = 0;
    if (!(ratio < R(3.0))) {
      const R lratio = lxi * delabm1 / (ratio * dlog(R(10)));
      laorb = laorb + lratio / z0noz;
      lz0noz = -lratio * aorb / (z0noz * z0noz);
    }
    if (!(a1 < a2)) { if (!(US < R(0.0001))) lUS = lUS - lz0noz * P_::RNUAIRM / (US * US); }
    else if (Z0 < R(0.0005)) lZ0 = lZ0 + lz0noz * R(0.04);
    luorbt = luorbt + lre * (R(4.0) / nu) * aorb;
    laorb = laorb + lre * (R(4.0) / nu) * uorbt;
    const R luo = luorbt / dsqrt(tiny + uo), lao = laorb / dsqrt(tiny + ao);
    s.for_bins(ml, [&](int m, int k) {
      const R sig = P_::ZPI * S.FR[m];
      LAM[k + ld * m] = LAM[k + ld * m] + (luo * S.DFIM[m] * (sig * sig) + lao * S.DFIM[m]);
    });
    lUS = lUS + lsig_n * dsig_us;
    lZ0 = lZ0 + lsig_n * dsig_z0;
    __syncwarp();
  }

  // The adjoints of both integral groups of one spectrum, unmasked (FMEAN,
  // AKMEAN) and masked by `mask` (FMEANWS), in one pass: the same sums and
  // terms as the two groups one after the other, LAM getting the unmasked
  // group's term first.
  __device__ void integrals_adj2(const R* Fs, const uint8_t* mask, R lfm, R lak, bool with_ak, R lfmw) const {
    const int kl = KL(), ml = ML(), ld = w.ld;
    const R DEL2 = dsqrt(P_::G) / P_::ZPI;
    R pe = 0, pf = 0, pa = 0, tail = 0, pe2 = 0, pf2 = 0, tail2 = 0;
    for (int m = lane; m < ml; m += 32) {
      R t = 0, t2 = 0;
      for (int k = 0; k < kl; ++k) {
        const int b = k + ld * m;
        const R v = Fs[b];
        t = t + v;
        if (mask[b]) t2 = t2 + v;
      }
      pe = pe + t * S.DFIM[m];
      pf = pf + t * S.DFIMOFR[m];
      if (with_ak) pa = pa + (T.shallow ? t / dsqrt(s.tfak(m)) * S.DFIM[m] : t * S.DFIMOFR[m] * DEL2);
      pe2 = pe2 + t2 * S.DFIM[m];
      pf2 = pf2 + t2 * S.DFIMOFR[m];
      if (m == ml - 1) { tail = t; tail2 = t2; }
    }
    pe = warp_sum(pe); pf = warp_sum(pf); pa = warp_sum(pa);
    pe2 = warp_sum(pe2); pf2 = warp_sum(pf2);
    tail = __shfl_sync(0xffffffffu, tail, (ml - 1) & 31);
    tail2 = __shfl_sync(0xffffffffu, tail2, (ml - 1) & 31);
    R lpe, lpf, lpa, ltail, lpe2, lpf2, lpa2, ltail2;
    integral_adj_terms(pe, pf, pa, tail, lfm, lak, with_ak, lpe, lpf, lpa, ltail);
    integral_adj_terms(pe2, pf2, R(0), tail2, lfmw, R(0), false, lpe2, lpf2, lpa2, ltail2);
    s.for_bins(ml, [&](int m, int k) {
      const int b = k + ld * m;
      R lt = lpe * S.DFIM[m] + lpf * S.DFIMOFR[m];
      if (with_ak) lt = lt + lpa * (T.shallow ? S.DFIM[m] / dsqrt(s.tfak(m)) : S.DFIMOFR[m] * DEL2);
      if (m == ml - 1) lt = lt + ltail;
      R v = LAM[b] + lt;
      if (mask[b]) {
        R lt2 = lpe2 * S.DFIM[m] + lpf2 * S.DFIMOFR[m];
        if (m == ml - 1) lt2 = lt2 + ltail2;
        v = v + lt2;
      }
      LAM[b] = v;
    });
    __syncwarp();
  }
  // The adjoints of the row-sum totals pe, pf, pa and of the tail row from
  // those of FMEAN (lfm) and AKMEAN (lak).
  __device__ void integral_adj_terms(R pe, R pf, R pa, R tail, R lfm, R lak, bool with_ak, R& lpe, R& lpf, R& lpa,
                                     R& ltail) const {
    const R DEL2 = dsqrt(P_::G) / P_::ZPI;
    const R e_raw = T.MO_TAIL * tail + pe, emean = dmax(e_raw, R(1.0E-12));
    const R den_raw = T.MM1_TAIL * tail + pf, den = dmax(den_raw, R(1.0E-12));
    R le = 0;
    lpe = 0; lpf = 0; lpa = 0; ltail = 0;
    if (with_ak && emean > R(1.0E-12)) {
      const R wm = T.MM1_TAIL * DEL2 * tail + pa, qv = emean / wm;
      const R lq = lak * R(2) * qv;
      le = le + lq / wm;
      const R lwm = -lq * emean / (wm * wm);
      lpa = lwm; ltail = ltail + lwm * T.MM1_TAIL * DEL2;
    }
    le = le + lfm / den;
    const R lden = -lfm * emean / (den * den);
    if (den_raw >= R(1.0E-12)) { lpf = lden; ltail = ltail + lden * T.MM1_TAIL; }
    if (e_raw >= R(1.0E-12)) { lpe = le; ltail = ltail + le * T.MO_TAIL; }
  }

  // F <- F0 (the input spectrum), read back from global memory.
  __device__ void reload_f0() const {
    const int kl = KL(), ld = w.ld;
    s.for_bins(ML(), [&](int m, int k) { w.F[k + ld * m] = __ldg(&F0g[ldg * (size_t)(k + kl * m)]); });
    __syncwarp();
  }

  // ---- ST6 (IPHYS = 2) ---------------------------------------------------------
  // Record of the LFACTOR iteration, at the end of the tape rows.
  __device__ R* lfrec() const { return AT + 14 * ML() - 16; }
  // dUSTAR/dU10 of W3FLX4 (:5372-5443); Z0 does not enter the step.
  __device__ R w3flx4_dus(R U) const {
    if (U >= R(50.33)) return R(0);
    const R cd = T.CDFAC * (R(8.058) + R(0.967) * U - R(0.016) * (U * U)) * R(1E-4);
    const R dcd = T.CDFAC * (R(0.967) - R(0.032) * U) * R(1E-4);
    const R sq = dsqrt(cd);
    return sq + U * dcd / (R(2) * sq);
  }

  // Forward ST6 step with recording (the forward kernel's statement order).
  __device__ void forward6() {
    const int ml = ML(), ld = w.ld;
    ju = min(300, max((int)lround((double)(s.U10 / T.DELU)), 1));
    R emean, emeanws;
    akmean = 0;
    const bool need_ak = T.shallow && T.isnonlin == 0;
    s.wavnu2();
    s.w3flx4(us1, z01);
    s.lfrec = lfrec();
    int nit = 0;
    R tail = 0, tailw = 0;
    s.llcopy = LL1;  // the first LLWS mask, kept for the reverse sweep
    s.sinput_st6(us1, tauw1, nit, tail, tailw, need_ak);
    s.lfrec = nullptr;
    s.llcopy = nullptr;
    phase();
    s.integral_sums(tail, tailw, emean, fmean, need_ak ? &akmean : nullptr, emeanws, fmeanws);
    mij = s.frcutindex_st6(fmean, us1);
    us2 = us1; z02 = z01;
    s.imphftail(mij);  // F = F1 from here on
    phase();
    s.sdissip_st6();
    phase();
    s.snonlin(akmean);
    phase();
    fmx = dmax(fmeanws, fmean);
    update_rows();
    mij2 = cutoff_after_update();
  }

  // SDISSIP_ST6^T and W3SWL6^T on F1 (:4929-5252): SL += (T12 + AB) F and
  // FL += T12 + AB per frequency row.  T12 = -(T1 + 7E-5 P) with P the prefix
  // sum over frequency (transposed: a suffix sum), AB = -2/3 b1 sig sqrt(BN)
  // with BN = sig WN^3 (row sum / narrowness sum) = sig WN^3 max_k a_k and b1
  // from the frequency-weighted total and the frozen MAXLOC row.
  __device__ void sdissip_st6_adj() const {
    const int kl = KL(), nk = ML(), ld = w.ld;
    s.wavnu2();
    const R* WN = w.t(0); const R* CG = w.t(1);
    R *T12 = w.t(2), *ABV = w.t(3), *LR = w.t(4), *LS = w.t(5), *LQ = w.t(6), *LADF = w.t(7);
    R *NEX = AT, *ADF = AT + nk, *SA = AT + 2 * nk, *KX = AT + 3 * nk, *BN = AT + 4 * nk, *ET = AT + 5 * nk;
    const R bnt = R(0.035) * R(0.035);
    const R xfac = (R(1.0) - R(1.0) / P_::CO) / (P_::CO - R(1.0) / P_::CO);
    R ps = 0, amax = -R(1);
    int imax = 0;
    for (int m = lane; m < nk; m += 32) {
      const R sig = P_::ZPI * S.FR[m];
      const R* fm = w.F + ld * m;
      const R2* lv = w.SF + ld * m;
      const R et = (P_::ZPI * bnt) / (CG[m] * (WN[m] * WN[m] * WN[m]));
      R sm = 0, lr = 0;
      for (int k = 0; k < kl; ++k) { sm = sm + fm[k]; lr = lr + (lv[k].x * fm[k] + lv[k].y); }
      LR[m] = lr;
      const R nex = dmax(R(0.0), sm * T.DELTH - et) / et;
      const R nex4 = (nex * nex) * (nex * nex);
      NEX[m] = nex; ET[m] = et;
      T12[m] = R(4.75E-6) * S.FR[m] * nex4;  // T1 until the scan
      const R dfii = (m > 0 && m < nk - 1) ? S.DF[m] * xfac : S.DF[m];
      ADF[m] = nex4 * dfii;
      const R cgs = CG[m] / (P_::ZPI * sig);
      R sa = 0, mx = 0;
      int kx = 0;
      for (int k = 0; k < kl; ++k) {
        const R a = fm[k] * cgs;
        sa = sa + a;
        if (k == 0 || mx < a) { mx = a; kx = k; }
      }
      R s2 = 0;
      if (mx < R(1.0E-34)) { s2 = R(kl); kx = -1; }
      else { const R rmx = R(1.) / mx; for (int k = 0; k < kl; ++k) s2 = s2 + (fm[k] * cgs) * rmx; }
      const R anar = R(1.0) / (s2 * T.DELTH);
      SA[m] = sa; KX[m] = R(kx);
      BN[m] = anar * (sa * sig * T.DELTH) * (WN[m] * WN[m] * WN[m]);
      ps = ps + sa * (P_::ZPI * S.DFIM[m] * sig) / CG[m];
      if (sa > amax) { amax = sa; imax = m; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const R oa = __shfl_xor_sync(0xffffffffu, amax, o);
      const int oi = __shfl_xor_sync(0xffffffffu, imax, o);
      if (oa > amax || (oa == amax && oi < imax)) { amax = oa; imax = oi; }
    }
    ps = warp_sum(ps);
    __syncwarp();
    const R b1 = R(0.0041) * (R(2.) * dsqrt(ps) * WN[imax]);
    // T2 prefix sum as the forward forms it, then the suffix sum of the
    // adjoints of P
    R carry = 0;
    for (int base = 0; base < nk; base += 32) {
      const int m = base + lane;
      R v = (m < nk) ? ADF[m] : R(0);
      for (int o = 1; o < 32; o <<= 1) { const R u = __shfl_up_sync(0xffffffffu, v, o); if (lane >= o) v = v + u; }
      v = v + carry;
      if (m < nk) {
        const R t1 = T12[m], p = R(7.00E-5) * v;
        T12[m] = R(-1.0) * (dmax(R(0.0), t1) + dmax(R(0.0), p));
        LADF[m] = (R(0.0) < p) ? -R(7.00E-5) * LR[m] : R(0);  // adjoint of P(m), before the suffix sum
      }
      carry = __shfl_sync(0xffffffffu, v, 31);
    }
    __syncwarp();
    R lb1 = 0;
    for (int m = lane; m < nk; m += 32) {
      const R sig = P_::ZPI * S.FR[m];
      R ab = 0;
      if (SA[m] > R(1.E-30)) {
        const R sb = dsqrt(BN[m]);
        ab = -(R(2.) / R(3.) * b1 * sig * sb);
        lb1 = lb1 + LR[m] * (-(R(2.) / R(3.)) * sig * sb);
        const R lbn = sb > R(0) ? LR[m] * (-(R(2.) / R(3.)) * b1 * sig) / (R(2) * sb) : R(0);
        LQ[m] = lbn * sig * (WN[m] * WN[m] * WN[m]);  // adjoint of sa/s2 (= max_k a_k)
      } else LQ[m] = R(0);
      ABV[m] = ab;
    }
    lb1 = warp_sum(lb1);
    const R lps = ps > R(0) ? lb1 * R(0.0041) * WN[imax] / dsqrt(ps) : R(0);
    __syncwarp();
    // suffix sums of the P adjoints (chunks from the top)
    R scarry = 0;
    for (int top = ((nk - 1) / 32) * 32; top >= 0; top -= 32) {
      const int m = top + lane;
      R v = (m < nk) ? LADF[m] : R(0);
      for (int o = 1; o < 32; o <<= 1) { const R u = __shfl_down_sync(0xffffffffu, v, o); if (lane + o < 32) v = v + u; }
      v = v + scarry;
      scarry = __shfl_sync(0xffffffffu, v, 0);
      __syncwarp();
      if (m < nk) LADF[m] = v;
    }
    __syncwarp();
    for (int m = lane; m < nk; m += 32) {
      const R sig = P_::ZPI * S.FR[m];
      const R dfii = (m > 0 && m < nk - 1) ? S.DF[m] * xfac : S.DF[m];
      const R lt1 = -LR[m];
      const R lnex4 = lt1 * R(4.75E-6) * S.FR[m] + LADF[m] * dfii;
      const R nex = NEX[m];
      LS[m] = nex > R(0) ? lnex4 * R(4) * (nex * nex * nex) * T.DELTH / ET[m] : R(0);
      // adjoint of the row sum sa: the frequency weights of b1, and the
      // narrowness factor when the row has no maximum
      R lsa = lps * (P_::ZPI * S.DFIM[m] * sig) / CG[m];
      if (KX[m] < R(0)) lsa = lsa + LQ[m] / R(kl);
      SA[m] = lsa;  // reused: adjoint of the row sum
    }
    __syncwarp();
    s.for_bins(nk, [&](int m, int k) {
      const int b = k + ld * m;
      const R sig = P_::ZPI * S.FR[m], cgs = CG[m] / (P_::ZPI * sig);
      R l = w.SF[b].x * (T12[m] + ABV[m]) + LS[m] + cgs * SA[m];
      if (KX[m] >= R(0) && k == (int)KX[m]) l = l + cgs * LQ[m];
      LAM[b] = LAM[b] + l;
    });
    __syncwarp();
  }

  // SINPUT_ST6^T with LFACTOR^T (:4465-4925) on F0.  The iteration's
  // decisions (its count, the sign sequence that fixes every DRTAU, the
  // MIN(1, EXP) branches, the reduce flag) are those of the forward pass, so
  // the final RTAU is the first one, ERR/90, times a constant, and LFACT
  // depends on the spectrum and u* through the first stress sums and through
  // its exponent.  In: SF = {lambda_SL, lambda_FL}, lTAUW.  Adds to LAM, lus
  // (adjoint of USTAR) and lU10 (tau_vis).
  __device__ void sinput_st6_adj(R lTAUW, R& lus, R& lU10) const {
    const int kl = KL(), nk = ML(), nk10 = T.NK10, ld = w.ld;
    s.wavnu2();
    const R* WN = w.t(0); const R* CG = w.t(1);
    R *SQB = w.t(2), *CI10 = w.t(3), *SDX = w.t(4), *SDY = w.t(5), *LF = w.t(6), *LLF = w.t(7);
    R *LSDX = AT, *LSDY = AT + nk10, *KXR = AT + 2 * nk10;
    const R* rec = lfrec();
    const R USTAR = us1, U10 = s.U10, ROAIRN = s.ROAIRN;
    const R cu = crcos(s.UDIR), su = crsin(s.UDIR), uproxy = R(32.) * USTAR;
    const R raw = ROAIRN / P_::ROWATER, gro = P_::G * P_::ROWATER;
    const int nit = (int)rec[LF_NIT];
    const bool reduce = rec[LF_REDUCE] != R(0);
    const R rl = rec[LF_RLAST];
    // growth rate of bin (m, k) and its parts
    struct Bin { R proj, w, th, g, d1, d2; bool up; };
    auto bin = [&](int m, int k) {
      Bin q;
      const R sig = P_::ZPI * S.FR[m], sqb = SQB[m];
      q.proj = rsub(rmul(uproxy * CI10[m], radd(rmul(S.COSTH[k], cu), rmul(S.SINTH[k], su))), R(1.));
      const R w1 = dmax(R(0.), q.proj), w2 = dmin(R(0.), q.proj);
      q.up = q.proj > R(0.);
      q.w = q.up ? w1 * w1 : w2 * w2;
      q.th = dtanh(rsub(rmul(R(10.) * sqb, q.w), R(11.)));
      q.g = R(2.8) - (R(1.) + q.th);
      q.d1 = q.up ? raw * sig * q.g * sqb * q.w : R(0.);
      q.d2 = q.up ? R(0.) : raw * sig * R(0.09) * q.g * sqb * q.w;
      return q;
    };
    // forward quantities per frequency (lane = m): SQB, CI10, the first
    // maximum of the row, and the directional stress sums
    for (int m = lane; m < nk; m += 32) {
      const R sig = P_::ZPI * S.FR[m];
      const R* fm = w.F + ld * m;
      const R zs = P_::ZPI * sig, cg = CG[m];
      const RecipDiv<R> qzs(zs);
      R sm = 0, mx = 0;
      int kx = 0;
      for (int k = 0; k < kl; ++k) {
        const R a = qzs(rmul(fm[k], cg));
        sm = sm + a;
        if (k == 0 || mx < a) { mx = a; kx = k; }
      }
      R s2 = 0;
      if (mx < R(1.0E-34)) { s2 = R(kl); kx = -1; }
      else {
        const RecipDiv<R> qmx(mx);
        for (int k = 0; k < kl; ++k) s2 = s2 + qmx(qzs(rmul(fm[k], cg)));
      }
      const R adensig = sm * sig * T.DELTH, anar = R(1.0) / (s2 * T.DELTH);
      SQB[m] = dsqrt(anar * adensig * (WN[m] * WN[m] * WN[m]));
      CI10[m] = WN[m] / sig;
      KXR[m] = R(kx);
    }
    __syncwarp();
    for (int m = lane; m < nk; m += 32) {
      const R sig = P_::ZPI * S.FR[m], zs = P_::ZPI * sig, cg = CG[m];
      const RecipDiv<R> qzs(zs), qcg(cg);
      const R* fm = w.F + ld * m;
      R bx = 0, by = 0;
      for (int k = 0; k < kl; ++k) {
        const Bin q = bin(m, k);
        const R a = qzs(rmul(fm[k], cg));
        const R sd = qcg(rmul(rmul(q.d1, a), sig));
        bx = radd(bx, rmul(dmax(R(0.), sd), S.COSTH[k]));
        by = radd(by, rmul(dmax(R(0.), sd), S.SINTH[k]));
      }
      SDX[m] = bx * T.DELTH; SDY[m] = by * T.DELTH;
    }
    __syncwarp();
    if (nk < nk10) {
      const R signk = S.SIG10[nk - 1];
      for (int i = nk + lane; i < nk10; i += 32) {
        const R r = (signk / S.SIG10[i]) * (signk / S.SIG10[i]);
        SDX[i] = SDX[nk - 1] * r; SDY[i] = SDY[nk - 1] * r;
        CI10[i] = S.SIG10[i] * R(0.101978);
      }
    }
    for (int i = lane; i < nk10; i += 32) {
      LF[i] = nit > 0 ? dmin(R(1.0), crexp(rmul(rsub(R(1.0), rmul(uproxy, CI10[i])), rl))) : R(1.0);
      LLF[i] = R(0);
    }
    __syncwarp();
    // 1. the bins: lambda of the total rate, of D1 and D2; LFACT's row adjoint.
    // Directions 0..31 go one frequency at a time; the directions beyond 32
    // of all frequencies in one pass, one lane per (frequency, direction),
    // their row-sum terms through XC (tape space free here).
    const int kmain = kl < 32 ? kl : 32, nx = kl - kmain;
    R* XC = AT + 3 * nk10;
    const bool bx = nx > 0 && 3 * nk10 + nk * nx <= 14 * nk - 16;
    auto body1 = [&](int m, int k) -> R {
      const int b = k + ld * m;
      const Bin q = bin(m, k);
      const R lfr = reduce ? LF[m] : R(1);
      const R dtot = q.d1 * lfr - q.d2;
      const R2 v = w.SF[b];
      const R f = w.F[b];
      const R ld_ = v.x * f + v.y;
      LAM[b] = LAM[b] + v.x * dtot;
      w.SF[b] = r2(ld_ * lfr, -ld_);  // {lambda_D1, lambda_D2}
      return reduce ? ld_ * q.d1 : R(0);
    };
    for (int m = 0; m < nk; ++m) {
      R llf = 0;
      if (bx) { if (lane < kmain) llf = body1(m, lane); }
      else for (int k = lane; k < kl; k += 32) llf = llf + body1(m, k);
      llf = warp_sum(llf);
      if (lane == 0) LLF[m] = llf;
    }
    if (bx) {
      for (int it = lane; it < nk * nx; it += 32) { const int m = it / nx; XC[it] = body1(m, kmain + it - m * nx); }
      __syncwarp();
      for (int m = lane; m < nk; m += 32) { R t = LLF[m]; for (int x = 0; x < nx; ++x) t = t + XC[m * nx + x]; LLF[m] = t; }
    }
    __syncwarp();
    // 2. the stress sums: final (after the iteration) and first
    const R tx = rec[LF_TX], ty = rec[LF_TY], tw = dsqrt(tx * tx + ty * ty);
    const R ltx = tw > R(0) ? lTAUW * tx / tw : R(0), lty = tw > R(0) ? lTAUW * ty / tw : R(0);
    const R* DS10 = S.DSII10;
    R ltx0 = 0, lty0 = 0, lustar = 0;
    if (nit > 0) {
      R lrl = 0, luq = 0;
      for (int i = lane; i < nk10; i += 32) {
        const R cd = gro * CI10[i] * DS10[i];
        const R llfi = LLF[i] + cd * (ltx * SDX[i] + lty * SDY[i]);
        LSDX[i] = cd * ltx * LF[i]; LSDY[i] = cd * lty * LF[i];
        const R qa = rsub(R(1.0), rmul(uproxy, CI10[i]));
        if (LF[i] < R(1.0)) {  // EXP branch of MIN(1, EXP(qa*rl))
          lrl = lrl + llfi * LF[i] * qa;
          luq = luq + llfi * LF[i] * rl * (-R(32.) * CI10[i]);
        }
      }
      lrl = warp_sum(lrl);
      lustar = lustar + warp_sum(luq);
      const R r0 = rec[LF_RTAU0], tau0 = rec[LF_TAU0], tt = rec[LF_TTOT];
      const R lr0 = r0 != R(0) ? lrl * (rl / r0) : R(0);
      const R lerr = lr0 / R(90.);
      const R ltau0 = lerr / tt;
      R ltt = -lerr * tau0 / (tt * tt);
      const R tvr = dmax(R(0.0), radd(-rmul(R(5.0E-5), U10), R(1.1E-3))) * (U10 * U10) * ROAIRN;
      const R tv = dmin(R(0.95) * tt, tvr);
      const R ax = radd(tv * cu, rec[LF_TX0]), ay = radd(tv * su, rec[LF_TY0]);
      const R lax = tau0 > R(0) ? ltau0 * ax / tau0 : R(0), lay = tau0 > R(0) ? ltau0 * ay / tau0 : R(0);
      ltx0 = lax; lty0 = lay;
      const R ltv = lax * cu + lay * su;
      if (tvr < R(0.95) * tt) {
        const R inner = radd(-rmul(R(5.0E-5), U10), R(1.1E-3));
        if (inner > R(0)) lU10 = lU10 + ltv * (-R(5.0E-5) * (U10 * U10) * ROAIRN + inner * R(2) * U10 * ROAIRN);
      } else ltt = ltt + R(0.95) * ltv;
      lustar = lustar + ltt * R(2) * USTAR * ROAIRN;
    } else {
      for (int i = lane; i < nk10; i += 32) { LSDX[i] = R(0); LSDY[i] = R(0); }
      ltx0 = ltx; lty0 = lty;
    }
    __syncwarp();
    for (int i = lane; i < nk10; i += 32) {
      const R cd = gro * CI10[i] * DS10[i];
      LSDX[i] = LSDX[i] + cd * ltx0; LSDY[i] = LSDY[i] + cd * lty0;
    }
    __syncwarp();
    if (nk < nk10) {  // the f^-2 extension carries SDX(NK) to 10 Hz
      const R signk = S.SIG10[nk - 1];
      R ex = 0, ey = 0;
      for (int i = nk + lane; i < nk10; i += 32) {
        const R r = (signk / S.SIG10[i]) * (signk / S.SIG10[i]);
        ex = ex + LSDX[i] * r; ey = ey + LSDY[i] * r;
      }
      ex = warp_sum(ex); ey = warp_sum(ey);
      if (lane == 0) { LSDX[nk - 1] = LSDX[nk - 1] + ex; LSDY[nk - 1] = LSDY[nk - 1] + ey; }
    }
    __syncwarp();
    // 3. the bins again: stress sums, growth-rate chain, narrowness (row sums
    // of the directions beyond 32 as in 1., in LSQ = the LLF row, free now)
    R luprox = 0;
    R* LSQ = LLF;
    auto body3 = [&](int m, int k) -> R {
      const R sig = P_::ZPI * S.FR[m], zs = P_::ZPI * sig, sqb = SQB[m];
      const R cg = CG[m], cgzs = cg / zs, sgcg = sig / cg;
      const RecipDiv<R> qzs(zs), qcg(cg);
      const R c1 = raw * sig;
      R lsqb = 0;
      {
        const int b = k + ld * m;
        const Bin q = bin(m, k);
        const R f = w.F[b];
        const R a = qzs(rmul(f, cg));
        const R sd = qcg(rmul(rmul(q.d1, a), sig));
        const R lsd = (R(0.) < sd) ? T.DELTH * (LSDX[m] * S.COSTH[k] + LSDY[m] * S.SINTH[k]) : R(0);
        const R2 v = w.SF[b];
        R ld1 = v.x + lsd * a * sgcg;
        const R la = lsd * q.d1 * sgcg;
        R lw = 0, lg = 0;
        if (q.up) {
          lg = ld1 * c1 * sqb * q.w;
          lsqb = lsqb + ld1 * c1 * q.g * q.w;
          lw = ld1 * c1 * q.g * sqb;
        } else {
          const R c2 = c1 * R(0.09);
          lg = v.y * c2 * sqb * q.w;
          lsqb = lsqb + v.y * c2 * q.g * q.w;
          lw = v.y * c2 * q.g * sqb;
        }
        const R lx = -lg * (R(1) - q.th * q.th);
        lsqb = lsqb + lx * R(10.) * q.w;
        lw = lw + lx * R(10.) * sqb;
        const R lproj = lw * R(2) * q.proj;
        luprox = luprox + lproj * CI10[m] * radd(rmul(S.COSTH[k], cu), rmul(S.SINTH[k], su));
        LAM[b] = LAM[b] + la * cgzs;
      }
      return lsqb;
    };
    for (int m = 0; m < nk; ++m) {
      R lsqb = 0;
      if (bx) { if (lane < kmain) lsqb = body3(m, lane); }
      else for (int k = lane; k < kl; k += 32) lsqb = lsqb + body3(m, k);
      lsqb = warp_sum(lsqb);
      if (lane == 0) LSQ[m] = lsqb;
    }
    if (bx) {
      for (int it = lane; it < nk * nx; it += 32) { const int m = it / nx; XC[it] = body3(m, kmain + it - m * nx); }
      __syncwarp();
      for (int m = lane; m < nk; m += 32) { R t = LSQ[m]; for (int x = 0; x < nx; ++x) t = t + XC[m * nx + x]; LSQ[m] = t; }
    }
    __syncwarp();
    // one lane per frequency: only the row's maximum bin (every bin of a row
    // without maximum) takes the narrowness term
    for (int m = lane; m < nk; m += 32) {
      const R sig = P_::ZPI * S.FR[m], zs = P_::ZPI * sig, sqb = SQB[m];
      const R cgzs = CG[m] / zs;
      const R lsqb = LSQ[m];
      // SQB = sqrt(sig WN^3 q) with q = row sum / narrowness sum (= the row's
      // first maximum of a, or the row sum / KL for an empty row)
      const R lq = sqb > R(0) ? lsqb * sig * (WN[m] * WN[m] * WN[m]) / (R(2) * sqb) : R(0);
      const int kx = (int)KXR[m];
      if (kx >= 0) LAM[kx + ld * m] = LAM[kx + ld * m] + lq * cgzs;
      else
        for (int k = 0; k < kl; ++k) LAM[k + ld * m] = LAM[k + ld * m] + (lq / R(kl)) * cgzs;
    }
    lustar = lustar + R(32.) * warp_sum(luprox);
    lus = lus + lustar;
    __syncwarp();
  }

  __device__ void reverse6(R lTAUW, R& lTAUW0, R& lU10) {
    imphftail_adj(mij2);
    R lus = 0, lfmx = 0;
    update_adj(lus, lfmx);
    phase();
    const R lak = snonlin_adj();
    phase();
    sdissip_st6_adj();
    phase();
    imphftail_adj(mij);
    reload_f0();
    lU10 = 0;
    sinput_st6_adj(lTAUW, lus, lU10);
    phase();
    R lfmean = 0, lfmeanws = 0;
    if (fmeanws < fmean) lfmean = lfmx; else lfmeanws = lfmx;
    integrals_adj2(w.F, LL1, lfmean, lak, T.shallow && T.isnonlin == 0, lfmeanws);
    lU10 = lU10 + w3flx4_dus(s.U10) * lus;
    lTAUW0 = R(0);  // ST6 overwrites TAUW: the input does not enter the step
  }

  // The whole reverse sweep.  In: LAM = adjoint of the output spectrum, lTAUW =
  // adjoint of the output TAUW.  Out: LAM = adjoint of the input spectrum,
  // lTAUW0 and lU10.
  __device__ void reverse(R TAUW0, R lTAUW, R& lTAUW0, R& lU10) {
    imphftail_adj(mij2);
    R lus2 = 0, lz02 = 0, lfmx = 0;
    update_adj(lus2, lfmx);
    phase();
    const R lak = snonlin_adj();
    phase();
    sdissip_adj();
    phase();
    stresso_adj(1, w.F, us2, z02, lTAUW, lus2, lz02);
    sinput_adj(1, w.F, us2, z02, w.SF, lus2, lz02);
    phase();
    imphftail_adj(mij);
    reload_f0();
    const adj::Jac2<R> J2 = airsea_jac(s.U10, tauw1);
    lU10 = J2.d00 * lus2 + J2.d10 * lz02;
    const R ltauw1 = J2.d01 * lus2 + J2.d11 * lz02;
    R lus1 = 0, lz01 = 0;
    stresso_adj(0, w.F, us1, z01, ltauw1, lus1, lz01);
    phase();
    sinput_adj(0, w.F, us1, z01, nullptr, lus1, lz01);
    phase();
    R lfmean = 0, lfmeanws = 0;
    if (fmeanws < fmean) lfmean = lfmx; else lfmeanws = lfmx;
    integrals_adj2(w.F, LL1, lfmean, lak, T.shallow && T.isnonlin == 0, lfmeanws);
    const adj::Jac2<R> J1 = airsea_jac(s.U10, TAUW0);
    lU10 = lU10 + J1.d00 * lus1 + J1.d10 * lz01;
    lTAUW0 = J1.d01 * lus1 + J1.d11 * lz01;
  }
};

}  // namespace wamgpu
