// C ABI of libwamgpu (declarations and reference citations in include/wamgpu.h).
#include <cuda_runtime.h>
#include <algorithm>
#include <climits>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include "../../include/wamgpu.h"
#include "wamgpu_config.hpp"
#include "spectral_tables.hpp"
#include "propargs.hpp"
#include "kernels.hpp"

using namespace wamgpu;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { if (p) cudaFree(p); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { if (p) cudaFree(p); }
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr; n = 0;
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e == cudaSuccess) n = bytes;
    return e;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

struct ImplBase {
  virtual ~ImplBase() {}
};

}  // namespace

struct wamgpu_ctx {
  Config cfg{};
  std::string err;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // host->device copies overlapped with the kernels of a host-buffer step
  cudaStream_t down_stream = nullptr;  // device->host copies of a host-buffer step
  std::vector<cudaEvent_t> xfer_ev;     // ordering events between the two streams
  int nsm = 148;
  int P = 8;  // sea points per IMPLSCH CTA
  // grid (reference convention, host)
  int nsea = 0, ny = 0, n_ext = 0;
  int halo = 0;  // largest |neighbour - point| over KLAT/KLON (sea point numbers)
  int own0 = 0, own1 = -1;  // sea points this context updates ([own0, own1); own1 < 0: all), the rest are halo
  std::vector<int> klat, klon, kfromij;
  std::vector<float> wlat, sinph, cosph, dellam;
  std::vector<float> depth, u, v;
  std::vector<int> indep;
  bool have_grid = false, prepared = false;
  bool wncg_valid = false;  // the WN/CG rows match the current depth
  int counter = 1; double total_cfl = 0, cfl_min = 0; int variant = 0;
  // test diagnostics of IMPLSCH's integer decisions (wamgpu_set_diagnostics)
  int* diag = nullptr;
  unsigned char* diag_ll = nullptr;
  int diag_ld = 0;
  int wind_nx = 0, wind_ny = 0, wind_equal = 0;  // wind input grid (wamgpu_set_wind_grid)
  std::unique_ptr<ImplBase> impl;
  // opt-in kernel timing: event pairs per kernel class (0 = PROPAGS, 1 = IMPLSCH)
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[2];
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
  // precision-specific part
  virtual ~wamgpu_ctx() {}
};

namespace {

template <typename R> struct Impl : ImplBase {
  TableSet<R> tab;
  DevTables<R> dt{};
  PropArgs<R> pa{};
  bool has_enh = false;  // MAKE_SHALLOW_SNL factors uploaded to `enh` ([ij + nsea*(mc-1)])
  DevBuf dwork, dmasks;  // work of the derivative kernels
  DevBuf ckpt;           // checkpoints of an assimilation window
  DevBuf wncg;           // ST6: WN and CG per (sea point, frequency), formed by wamgpu_prepare_source
  int nckpt = 0, ckpt_ld = 0;
  DevBuf small, ismall, tfak, tcgond, tsihkd, flminfr, enh, gom, fr, sinth, costh;
  DevBuf outtab;         // integrated output: DFIM_FR, DFIM_FR2, MEANSQS deep-water weights, C (ML each)
  DevBuf ustar_max;      // MAXVAL(USTAR) word of the output step
  DevBuf wind_tab, wind_w;  // INTERPOLATION_TO_GRID tables (I1, I2, K1, K2; DI, DK) of the sea points
  DevBuf rst_stage, rst_perm;  // restart records: REAL staging chunk, IJ2NEWIJ
  DevBuf diamc;          // per-MC DIA rows and write masks (DevTables::diamc)
  DevBuf dslot;          // DIA batch slot entries (DevTables::dslot)
  // per-point metadata
  DevBuf d_klat, d_klon, d_wlat, d_dpsn, d_della0, d_drgm, d_indep, d_indep_g, d_ddphi, d_ddlam, d_duphi, d_dulam,
      d_dvphi, d_dvlam, d_u, d_v, d_depth;
  // model state used by the host-buffer entry points
  DevBuf fl3, scratch, u10, udir, tauw, ustar, z0, roairn, wstar, fluxes, status, cflext;
  std::vector<R> dco, dpsn;  // host
};

struct TimedLaunch {
  wamgpu_ctx* ctx; int cls; cudaStream_t s; std::pair<cudaEvent_t, cudaEvent_t> e{nullptr, nullptr};
  TimedLaunch(wamgpu_ctx* c, int k, cudaStream_t st) : ctx(c), cls(k), s(st) {
    if (!ctx->timing) return;
    if (ctx->ev_pool.empty()) {
      cudaEvent_t a, b;
      cudaEventCreate(&a); cudaEventCreate(&b);
      ctx->ev_pool.push_back({a, b});
    }
    e = ctx->ev_pool.back(); ctx->ev_pool.pop_back();
    cudaEventRecord(e.first, s);
  }
  ~TimedLaunch() {
    if (!e.first) return;
    cudaEventRecord(e.second, s);
    ctx->ev[cls].push_back(e);
  }
};

int fail(wamgpu_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}
int cuda_fail(wamgpu_ctx* c, cudaError_t e, const char* where) {
  return fail(c, WAMGPU_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define CK(call, where)                                 \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
  } while (0)

template <typename T> cudaError_t upload(DevBuf& b, const std::vector<T>& h, cudaStream_t s) {
  cudaError_t e = b.ensure(h.size() * sizeof(T) + 16);
  if (e != cudaSuccess) return e;
  if (h.empty()) return cudaSuccess;
  return cudaMemcpyAsync(b.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

template <typename R> int build_tables(wamgpu_ctx* ctx, Impl<R>& I) {
  const Config& c = ctx->cfg;
  TableSet<R>& t = I.tab;
  t.build(c);
  // packed small tables
  SmallLayout L{};
  std::vector<R> sr;
  auto putr = [&](int& off, const std::vector<R>& v) { off = (int)sr.size(); sr.insert(sr.end(), v.begin(), v.end()); };
  std::vector<R> delfl(t.ML);
  for (int m = 0; m < t.ML; ++m) delfl[m] = R(5.0E-07) * Phys<R>::G / powi(t.FR[m], 4) * R(c.idelt);
  // ST6 frequency axis extended to 10 Hz and its bandwidths (LFACTOR :4554-4599)
  int nk10;
  {
    const R sig1 = Phys<R>::ZPI * t.FR[0];
    nk10 = (int)std::ceil(std::log(R(10.) / (sig1 / Phys<R>::ZPI)) / std::log(Phys<R>::CO)) + 1;
    nk10 = std::max(t.ML, nk10);
  }
  std::vector<R> sig10(nk10), dsii10(nk10);
  {
    const R co = Phys<R>::CO, sig1 = Phys<R>::ZPI * t.FR[0];
    if (t.ML < nk10) {
      for (int i = 0; i < nk10; ++i) sig10[i] = sig1 * std::pow(co, R(i + 1) - R(1.0));
      for (int i = 0; i < nk10; ++i) dsii10[i] = R(0.5) * sig10[i] * (co - R(1.0) / co);
      dsii10[0] = R(0.5) * sig10[0] * (co - R(1.0));
      dsii10[nk10 - 1] = R(0.5) * sig10[nk10 - 1] * (co - R(1.0)) / co;
    } else {
      for (int i = 0; i < nk10; ++i) { sig10[i] = Phys<R>::ZPI * t.FR[i]; dsii10[i] = Phys<R>::ZPI * t.DF[i]; }
    }
  }
  putr(L.FR, t.FR); putr(L.DF, t.DF); putr(L.DFIM, t.DFIM); putr(L.DFIMOFR, t.DFIMOFR); putr(L.FR5, t.FR5);
  putr(L.FRM5, t.FRM5); putr(L.RHOWG_DFIM, t.RHOWG_DFIM); putr(L.TH, t.TH); putr(L.COSTH, t.COSTH);
  putr(L.SINTH, t.SINTH); putr(L.DELFL, delfl); putr(L.AF11, t.AF11);
  {  // RNLCOEF regrouped (rnl_slot), each MC's block 16-byte aligned
    std::vector<R> rn((size_t)RNL_STRIDE * t.MLSTHG, R(0));
    for (int mc = 0; mc < t.MLSTHG; ++mc)
      for (int i = 0; i < 25; ++i) rn[(size_t)RNL_STRIDE * mc + rnl_slot(i)] = t.RNLCOEF[25 * mc + i];
    while (sr.size() % 4) sr.push_back(R(0));
    putr(L.RNLCOEF, rn);
  }
  putr(L.SATW, t.SATWEIGHTS); putr(L.WTAUHF, t.WTAUHF); putr(L.SWELLFT, t.SWELLFT);
  putr(L.SIG10, sig10); putr(L.DSII10, dsii10);
  L.nreal = (int)sr.size();
  std::vector<int> si;
  auto puti = [&](int& off, const std::vector<int>& v) { off = (int)si.size(); si.insert(si.end(), v.begin(), v.end()); };
  puti(L.K1W, t.K1W); puti(L.K2W, t.K2W); puti(L.K11W, t.K11W); puti(L.K21W, t.K21W); puti(L.INLCOEF, t.INLCOEF);
  puti(L.IKP, t.IKP); puti(L.IKP1, t.IKP1); puti(L.IKM, t.IKM); puti(L.IKM1, t.IKM1); puti(L.INDSAT, t.INDICESSAT);
  L.nint = (int)si.size();
  cudaStream_t s = ctx->stream;
  CK(upload(I.small, sr, s), "upload tables");
  CK(upload(I.ismall, si, s), "upload tables");
  CK(upload(I.tfak, t.TFAK, s), "upload tables");
  CK(upload(I.tcgond, t.TCGOND, s), "upload tables");
  CK(upload(I.tsihkd, t.TSIHKD, s), "upload tables");
  CK(upload(I.flminfr, t.FLMINFR, s), "upload tables");
  CK(upload(I.gom, t.GOM, s), "upload tables");
  CK(upload(I.fr, t.FR, s), "upload tables");
  CK(upload(I.sinth, t.SINTH, s), "upload tables");
  CK(upload(I.costh, t.COSTH, s), "upload tables");
  {
    // MEANSQS deep-water weights FD(M) = DFIM(M)*(ZPI*FR(M))**4/G**2 (wam_interface_module.f90:721)
    std::vector<R> ot(t.DFIM_FR);
    ot.insert(ot.end(), t.DFIM_FR2.begin(), t.DFIM_FR2.end());
    for (int m = 0; m < t.ML; ++m)
      ot.push_back(t.DFIM[m] * powi(Phys<R>::ZPI * t.FR[m], 4) / powi(Phys<R>::G, 2));
    ot.insert(ot.end(), t.C.begin(), t.C.end());  // deep-water phase speeds (swell separation)
    CK(upload(I.outtab, ot, s), "upload tables");
  }
  DevTables<R>& d = I.dt;
  d.KL = t.KL; d.ML = t.ML; d.NS = t.KL * t.ML; d.NDEPTH = t.NDEPTH; d.MFRSTLW = t.MFRSTLW; d.MLSTHG = t.MLSTHG;
  d.KFRH = t.KFRH; d.NSDSNTH = t.NSDSNTH;
  d.NK10 = nk10;
  d.ld = t.KL | 1;
  d.scr = (std::max(std::max(t.ML, t.KL), nk10) + 31) / 32 * 32;
  d.need_sp = c.lcflx ? 1 : 0;
  // The DIA forms the interactions of the directions beyond the first 32
  // (NX = KL - 32) for a batch of consecutive MCs in one pass.  The batch's
  // slots take 8*NX reals per MC of scratch after the 8*KL of the per-MC
  // buffer, and the batch updates its target rows one kind (MC, MM, MM1, MP,
  // MP1) at a time, so the rows that one kind writes must be distinct within
  // a batch: strictly increasing in MC.  Otherwise the batch is one MC.
  d.dia_batch = 1;
  // Scratch rows 4 reals longer than a multiple of 32: the rows that lanes
  // read side by side in the ordered sums (the spectral integrals, TAUWINDS)
  // then start in different shared-memory banks.
  d.scr += 4;
  if (t.KL > 32) {
    const int nx = t.KL - 32, ML = t.ML, mfr1 = -t.MFRSTLW + 1, mfrl = ML - t.KFRH + mfr1;
    int b = 32 / nx;
    while (b > 1 && 8 * t.KL + 8 * nx * b > 8 * d.scr) --b;
    if (8 * t.KL + 8 * nx * b > 8 * d.scr) d.scr = ((8 * t.KL + 8 * nx * b + 7) / 8 + 31) / 32 * 32 + 4;
    int last[5] = {INT_MIN, INT_MIN, INT_MIN, INT_MIN, INT_MIN};
    bool mono = true;
    for (int mc = 1; mc <= t.MLSTHG; ++mc) {
      const int i = mc - t.MFRSTLW, MP = t.IKP[i], MP1 = t.IKP1[i], MM = t.IKM[i], MM1 = t.IKM1[i];
      const int regime = (mc > mfr1 && mc < mfrl) ? 0 : (mc >= mfrl ? 1 : 2);
      const bool wr[5] = {regime != 1 || (MM1 <= ML && mc <= ML), regime != 2,
                          regime == 0 || (regime == 1 && MM1 <= ML) || (regime == 2 && MM1 >= 1),
                          regime != 1 || (MM1 <= ML && mc <= ML && MP <= ML),
                          regime != 1 || (MM1 <= ML && mc <= ML && MP <= ML && MP1 <= ML)};
      const int row[5] = {mc, MM, MM1, MP, MP1};
      for (int q = 0; q < 5; ++q)
        if (wr[q]) {
          if (row[q] <= last[q]) mono = false;
          last[q] = row[q];
        }
    }
    if (!mono) b = 1;
    const int nbatch = (t.MLSTHG + b - 1) / b;
    d.dia_batch = nbatch > 0 ? (t.MLSTHG + nbatch - 1) / nbatch : 1;  // the same batch count, evenly filled
  }
  // The DIA^T batches the same directions but adds to the gathered rows (IC,
  // IP, IP1, IM, IM1 of INLCOEF), which repeat where they are clamped to the
  // ends of the spectrum.  A batch holds at most as many MCs as its slots
  // (4*NX reals each after the 6*KL of the per-MC buffer) and the lanes allow,
  // and a new batch starts wherever a kind's row equals the previous MC's.
  d.dia_adj_starts[0] = d.dia_adj_starts[1] = ~0ull;
  if (t.KL > 32) {
    const int nx = t.KL - 32;
    const int bmax = std::max(1, std::min(32 / nx, (8 * d.scr - 6 * t.KL) / (4 * nx)));
    d.dia_adj_starts[0] = d.dia_adj_starts[1] = 0;
    int nb = 0;
    for (int mc = 1; mc <= t.MLSTHG && mc <= 128; ++mc) {
      bool cut = nb == 0 || nb == bmax;
      if (!cut)
        for (int q = 0; q < 5; ++q) cut = cut || t.INLCOEF[5 * (mc - 1) + q] == t.INLCOEF[5 * (mc - 2) + q];
      if (cut) { d.dia_adj_starts[(mc - 1) >> 6] |= 1ull << ((mc - 1) & 63); nb = 0; }
      ++nb;
    }
  }
  d.iphys = c.iphys; d.shallow = c.shallow_run; d.isnonlin = c.isnonlin; d.lcflx = c.lcflx;
  d.DELTH = t.DELTH; d.DELTR = t.DELTR; d.INV_LOG_CO = t.INV_LOG_CO; d.MO_TAIL = t.MO_TAIL; d.MM1_TAIL = t.MM1_TAIL;
  d.DELU = t.DELU; d.DAL1 = t.DAL1; d.DAL2 = t.DAL2; d.X0TAUHF = t.X0TAUHF;
  d.BETAMAX = R(c.betamax); d.ZALP = R(c.zalp); d.ALPHA = R(c.alpha); d.TAUWSHELTER = R(c.tauwshelter);
  d.CDFAC = R(c.cdfac); d.DELT = R(c.idelt);
  d.lay = L;
  d.small = I.small.template as<R>(); d.ismall = I.ismall.template as<int>();
  d.TFAK = I.tfak.template as<R>(); d.TCGOND = I.tcgond.template as<R>(); d.FLMINFR = I.flminfr.template as<R>();
  if (d.NK10 > MAX_NK10) return fail(ctx, WAMGPU_E_ARG, "frequency grid too low: 10 Hz extension exceeds kernel bound");
  // every DIA gather row and scatter target the kernel can touch lies inside the spectrum
  {
    const int ML = t.ML, KL = t.KL, mfr1 = -t.MFRSTLW + 1, mfrl = ML - t.KFRH + mfr1;
    for (int v : t.K1W) if (v < 1 || v > KL) return fail(ctx, WAMGPU_E_ARG, "DIA angular index out of range");
    for (int v : t.K2W) if (v < 1 || v > KL) return fail(ctx, WAMGPU_E_ARG, "DIA angular index out of range");
    for (int v : t.K11W) if (v < 1 || v > KL) return fail(ctx, WAMGPU_E_ARG, "DIA angular index out of range");
    for (int v : t.K21W) if (v < 1 || v > KL) return fail(ctx, WAMGPU_E_ARG, "DIA angular index out of range");
    // the kernel forms partner and source directions as rotations of k by a
    // constant per table and KH: each table must be one
    for (const std::vector<int>* tb : {&t.K1W, &t.K2W, &t.K11W, &t.K21W})
      for (int kh = 0; kh < 2; ++kh) {
        const int off = ((*tb)[KL * kh] - 1) % KL;
        for (int k = 0; k < KL; ++k)
          if ((*tb)[k + KL * kh] - 1 != (k + off) % KL)
            return fail(ctx, WAMGPU_E_ARG, "DIA angular partner table is not a rotation of the directions");
      }
    for (int v : t.INLCOEF) if (v < 1 || v > ML) return fail(ctx, WAMGPU_E_ARG, "DIA frequency index out of range");
    for (int v : t.INDICESSAT) if (v < 1 || v > KL) return fail(ctx, WAMGPU_E_ARG, "saturation index out of range");
    auto in = [&](int m) { return m >= 1 && m <= ML; };
    for (int mc = 1; mc <= t.MLSTHG; ++mc) {
      int i = mc - t.MFRSTLW, MP = t.IKP[i], MP1 = t.IKP1[i], MM = t.IKM[i], MM1 = t.IKM1[i];
      bool ok = true;
      if (mc > mfr1 && mc < mfrl) ok = in(mc) && in(MM) && in(MM1) && in(MP) && in(MP1);
      else if (mc >= mfrl) ok = in(MM) && (MM1 > ML || (in(MM1) && (mc > ML || (in(mc) && (MP > ML || (in(MP) && (MP1 > ML || in(MP1))))))));
      else ok = (MM1 < 1 || in(MM1)) && in(mc) && in(MP) && in(MP1);
      if (!ok) return fail(ctx, WAMGPU_E_ARG, "DIA scatter target outside the spectrum");
      // the kernel updates the rows MC, MM, MM1, MP, MP1 of one phase without
      // ordering between them: they must be distinct
      int rows[5] = {mc, MM, MM1, MP, MP1};
      for (int x = 0; x < 5; ++x)
        for (int y = x + 1; y < 5; ++y)
          if (rows[x] == rows[y] && in(rows[x]) && in(rows[y]))
            return fail(ctx, WAMGPU_E_ARG, "DIA target rows coincide; unsupported frequency ratio");
    }
  }
  // Per-MC DIA bookkeeping, point-independent, as the kernels read it: three
  // int4 per MC = {IC, IP, IP1, IM} and {IM1, MC, MM, MM1} row offsets (the
  // gathered rows of INLCOEF, the target rows; row 0 where not written), then
  // {MP, MP1} offsets, the write flags (1 MC, 2 MM, 4 MM1, 8 MP, 16 MP1; 32 =
  // interior MC, FTAIL 1) and the AF11 index.  The regimes follow the
  // interior (:2890), high-tail (:2942) and low-tail (:2999) branches.
  {
    const int ML = t.ML, ld = d.ld, mfr1 = -t.MFRSTLW + 1, mfrl = ML - t.KFRH + mfr1;
    std::vector<int> dm((size_t)12 * std::max(1, t.MLSTHG), 0);
    for (int mc = 1; mc <= t.MLSTHG; ++mc) {
      const int im = mc - t.MFRSTLW, MP = t.IKP[im], MP1 = t.IKP1[im], MM = t.IKM[im], MM1 = t.IKM1[im];
      const int* ic5 = &t.INLCOEF[5 * (mc - 1)];
      const int regime = (mc > mfr1 && mc < mfrl) ? 0 : (mc >= mfrl ? 1 : 2);
      const bool wMM = regime != 2, wMM1 = regime == 0 || (regime == 1 && MM1 <= ML) || (regime == 2 && MM1 >= 1);
      const bool wMC = regime != 1 || (MM1 <= ML && mc <= ML);
      const bool wMP = regime != 1 || (MM1 <= ML && mc <= ML && MP <= ML);
      const bool wMP1 = regime != 1 || (MM1 <= ML && mc <= ML && MP <= ML && MP1 <= ML);
      int* e = &dm[(size_t)12 * (mc - 1)];
      for (int q = 0; q < 5; ++q) e[q] = ld * (ic5[q] - 1);
      e[5] = wMC ? ld * (mc - 1) : 0; e[6] = wMM ? ld * (MM - 1) : 0; e[7] = wMM1 ? ld * (MM1 - 1) : 0;
      e[8] = wMP ? ld * (MP - 1) : 0; e[9] = wMP1 ? ld * (MP1 - 1) : 0;
      e[10] = (wMC ? 1 : 0) | (wMM ? 2 : 0) | (wMM1 ? 4 : 0) | (wMP ? 8 : 0) | (wMP1 ? 16 : 0) | (regime == 0 ? 32 : 0);
      e[11] = im;
    }
    CK(upload(I.diamc, dm, ctx->stream), "upload tables");
    d.diamc = I.diamc.template as<int4>();
  }
  // DIA batch slots (KL > 32, NX = KL - 32 directions per MC of a batch).
  // Entry i < 4*NX of a slot, as int4: where the per-MC pass copies it in the
  // buffer, and the two buffer entries whose sum (over KH) the columns
  // 32..KL-1 gather through one partner table, then 0.  Entry i = (table q,
  // direction 32 + x) with q = i / NX.  The forward's buffer is {XM | XP}
  // [kh][k] (q: K2W, K21W read XM; K1W, K11W read XP); the adjoint's is
  // {XS | XM} (q: K1W, K11W read XS; K2W, K21W read XM).  A source column is
  // the target column rotated back by the table's offset.
  {
    const int KL = t.KL, nx = KL > 32 ? KL - 32 : 0;
    std::vector<int> ds((size_t)32 * std::max(1, nx), 0);
    auto rot = [KL](int k, int o) { const int v = k + o; return v >= KL ? v - KL : v; };
    auto put = [&](int e, const std::vector<int>* const tabs[4], int i) {
      const int q = i / nx, j = 32 + (i - q * nx), kh = q & 1, base = q < 2 ? 0 : 2 * KL;
      const std::vector<int>& tb = *tabs[q];
      int* v = &ds[(size_t)4 * e];
      v[0] = (q >> 1) * 2 * KL + kh * KL + j;
      v[1] = base + rot(j, KL - (tb[0] - 1));
      v[2] = base + KL + rot(j, KL - (tb[KL] - 1));
    };
    const std::vector<int>* const fw[4] = {&t.K2W, &t.K21W, &t.K1W, &t.K11W};
    const std::vector<int>* const ad[4] = {&t.K1W, &t.K11W, &t.K2W, &t.K21W};
    for (int i = 0; i < 4 * nx; ++i) { put(i, fw, i); put(4 * nx + i, ad, i); }
    CK(upload(I.dslot, ds, ctx->stream), "upload tables");
    d.dslot = I.dslot.template as<int4>();
  }
  // CTA shape: the number of sea points per CTA that keeps the most warps
  // resident per SM under the shared-memory budget (ties go to larger CTAs,
  // whose spectrum loads use longer contiguous runs)
  int dev = c.device;
  int maxsm = 0, smpersm = 0;
  CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "device attribute");
  CK(cudaDeviceGetAttribute(&smpersm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev), "device attribute");
  const int choices_f[3] = {8, 6, 4}, choices_d[2] = {4, 2};
  const int* choices = sizeof(R) == 4 ? choices_f : choices_d;
  const int nchoice = sizeof(R) == 4 ? 3 : 2;
  ctx->P = 0;
  int best_warps = 0;
  for (int q = 0; q < nchoice; ++q) {
    int P = choices[q];
    size_t need = implsch_smem_bytes(d, P);
    if ((int)need > maxsm) continue;
    int ctas = std::min(32 / P, (int)(smpersm / (need + 1024)));
    if (P * ctas > best_warps) { best_warps = P * ctas; ctx->P = P; }
  }
  if (ctx->P) CK(implsch_set_max_smem<R>(ctx->P, implsch_smem_bytes(d, ctx->P)), "smem attribute");
  if (!ctx->P) return fail(ctx, WAMGPU_E_ARG, "spectrum too large for the shared-memory workspace");
  CK(cudaStreamSynchronize(s), "table upload");
  return WAMGPU_OK;
}

template <typename R> R rf(float x) { return R(x); }

// PREPARE_PROPAGATION host part: INDEP, DCO/DPSN, gradients, INDEP_G and
// the variant metric factors; the coefficients themselves live in the kernels.
template <typename R> int prepare_prop(wamgpu_ctx* ctx, Impl<R>& I, float* total_cfl, int* counter) {
  const Config& c = ctx->cfg;
  const TableSet<R>& t = I.tab;
  const int n = ctx->nsea, KL = t.KL, ML = t.ML, ND = t.NDEPTH;
  auto KLAT = [&](int ij1, int ic, int j) { return ctx->klat[(ij1 - 1) + n * ((ic - 1) + 2 * (j - 1))]; };
  auto KLON = [&](int ij1, int d) { return ctx->klon[(ij1 - 1) + n * (d - 1)]; };
  auto WLAT = [&](int ij1, int ic) { return R(ctx->wlat[(ij1 - 1) + n * (ic - 1)]); };
  std::vector<R> D(n + 1, R(999.0)), U(n + 1, R(0)), V(n + 1, R(0));
  for (int i = 0; i < n; ++i) { D[i + 1] = R(ctx->depth[i]); U[i + 1] = R(ctx->u[i]); V[i + 1] = R(ctx->v[i]); }
  // INDEP (:327-332)
  ctx->indep.assign(n, 1);
  if (c.shallow_run)
    for (int i = 0; i < n; ++i) {
      int v = f_nint(std::log(D[i + 1] / t.DEPTHA) / std::log(t.DEPTHD) + R(1.));
      ctx->indep[i] = std::min(std::max(v, 1), ND);
    }
  const bool refr = c.refraction_d_run || c.refraction_c_run;
  // GRADIENT (:182-275) on 1-based fields with land slot 0
  const R delphi = R(c.delphi);
  auto gradient = [&](const std::vector<R>& Fd, std::vector<R>& dlat, std::vector<R>& dlon) {
    dlat.assign(n, R(0)); dlon.assign(n, R(0));
    for (int ij = 1; ij <= n; ++ij) {
      int ip = KLAT(ij, 2, 1), im = KLAT(ij, 1, 1);
      if (c.reduced_grid) {
        int ip2 = KLAT(ij, 2, 2), im2 = KLAT(ij, 1, 2);
        if (ip && im && ip2 && im2)
          dlat[ij - 1] = (WLAT(ij, 2) * Fd[ip] + (R(1.) - WLAT(ij, 2)) * Fd[ip2] - WLAT(ij, 1) * Fd[im] -
                          (R(1.) - WLAT(ij, 1)) * Fd[im2]) / (R(2.) * delphi);
        else if (ip && im) dlat[ij - 1] = (Fd[ip] - Fd[im]) / (R(2.) * delphi);
        else if (ip2 && im2) dlat[ij - 1] = (Fd[ip2] - Fd[im2]) / (R(2.) * delphi);
      } else if (ip && im) dlat[ij - 1] = (Fd[ip] - Fd[im]) / (R(2.) * delphi);
      int ie = KLON(ij, 2), iw = KLON(ij, 1);
      if (ie && iw) dlon[ij - 1] = (Fd[ie] - Fd[iw]) / (R(2.) * R(ctx->dellam[ctx->kfromij[ij - 1] - 1]));
    }
  };
  std::vector<R> ddphi(n, 0), ddlam(n, 0), duphi(n, 0), dulam(n, 0), dvphi(n, 0), dvlam(n, 0);
  std::vector<int> indep_g(n, 1);
  if (refr) {
    if (c.shallow_run) {
      gradient(D, ddphi, ddlam);
      if (c.spherical_run) for (int i = 0; i < n; ++i) ddlam[i] = ddlam[i] * I.dco[i + 1];
    }
    if (c.refraction_c_run) {
      gradient(U, duphi, dulam); gradient(V, dvphi, dvlam);
      if (c.spherical_run)
        for (int i = 0; i < n; ++i) { dulam[i] = dulam[i] * I.dco[i + 1]; dvlam[i] = dvlam[i] * I.dco[i + 1]; }
    }
    if (c.shallow_run)  // INDEP_G (:413-475)
      for (int ij = 1; ij <= n; ++ij) {
        R dm = R(4.) * D[ij]; int iz = 4;
        int ip = KLAT(ij, 2, 1), im = KLAT(ij, 1, 1);
        if (c.reduced_grid) {
          int ip2 = KLAT(ij, 2, 2), im2 = KLAT(ij, 1, 2);
          if (ip && im && ip2 && im2) {
            dm = dm + WLAT(ij, 2) * D[ip] + (R(1.) - WLAT(ij, 2)) * D[ip2] + WLAT(ij, 1) * D[im] + (R(1.) - WLAT(ij, 1)) * D[im2];
            iz += 2;
          } else if (ip && im) { dm = dm + D[ip] + D[im]; iz += 2; }
          else if (ip2 && im2) { dm = dm + D[ip2] + D[im2]; iz += 2; }
        } else if (ip && im) { dm = dm + D[ip] + D[im]; iz += 2; }
        int ie = KLON(ij, 2), iw = KLON(ij, 1);
        if (ie && iw) { dm = dm + D[ie] + D[iw]; iz += 2; }
        dm = dm / R(iz);
        int v = f_nint(std::log(dm / t.DEPTHA) / std::log(t.DEPTHD) + R(1.));
        indep_g[ij - 1] = std::min(std::max(v, 1), ND);
      }
  }
  // variant and metric factors (PREPARE_PROPAGATION_COEF :837-917)
  int var;
  if (!c.spherical_run) var = c.refraction_c_run ? (c.shallow_run ? V_CART_SHALLOW_CUR : V_CART_DEEP_CUR) : (c.shallow_run ? V_CART_SHALLOW : V_CART_DEEP);
  else var = c.refraction_c_run ? (c.shallow_run ? V_SPHER_SHALLOW_CURR : V_SPHER_DEEP_CURR) : (c.shallow_run ? V_SPHER_SHALLOW : V_SPHER_DEEP);
  ctx->variant = var;
  const R delpro = R(c.idelpro);
  std::vector<R> della0(n), drgm(n, R(0));
  for (int i = 0; i < n; ++i) {
    R dl = R(ctx->dellam[ctx->kfromij[i] - 1]);
    if (var == V_CART_DEEP) della0[i] = delpro / dl;
    else if (var == V_SPHER_DEEP) della0[i] = delpro * I.dco[i + 1] / dl;
    else if (c.spherical_run) della0[i] = R(0.5) * delpro * I.dco[i + 1] / dl;
    else della0[i] = R(0.5) * delpro / dl;
    if (c.spherical_run) drgm[i] = R(ctx->sinph[ctx->kfromij[i] - 1]) * I.dco[i + 1];
  }
  PropArgs<R>& A = I.pa;
  A.nsea = n; A.KL = KL; A.ML = ML; A.variant = var; A.reduced = c.reduced_grid; A.refr_d = c.refraction_d_run;
  A.spherical = c.spherical_run; A.counter = 1; A.rcounter = R(1); A.NDEPTH = ND;
  A.i0 = ctx->own0; A.i1 = ctx->own1 < 0 ? n : ctx->own1;
  A.DELPH0 = (var == V_CART_DEEP) ? delpro / delphi : R(0.5) * delpro / delphi;
  A.DELTH0 = R(0.5) * delpro / t.DELTR;
  A.DELTHR = R(0.5) * delpro / t.DELTH;
  A.DELFR0 = c.shallow_run ? R(0.5) * delpro / (R(0.1) * Phys<R>::ZPI) : R(0.5) * delpro * R(2.1) / R(0.2);
  cudaStream_t s = ctx->stream;
  std::vector<R> wl(ctx->wlat.begin(), ctx->wlat.end());
  CK(upload(I.d_klat, ctx->klat, s), "upload grid");
  CK(upload(I.d_klon, ctx->klon, s), "upload grid");
  CK(upload(I.d_wlat, wl, s), "upload grid");
  CK(upload(I.d_dpsn, I.dpsn, s), "upload grid");
  CK(upload(I.d_della0, della0, s), "upload grid");
  CK(upload(I.d_drgm, drgm, s), "upload grid");
  CK(upload(I.d_indep, ctx->indep, s), "upload grid");
  CK(upload(I.d_indep_g, indep_g, s), "upload grid");
  CK(upload(I.d_ddphi, ddphi, s), "upload grid"); CK(upload(I.d_ddlam, ddlam, s), "upload grid");
  CK(upload(I.d_duphi, duphi, s), "upload grid"); CK(upload(I.d_dulam, dulam, s), "upload grid");
  CK(upload(I.d_dvphi, dvphi, s), "upload grid"); CK(upload(I.d_dvlam, dvlam, s), "upload grid");
  std::vector<R> uu(U.begin() + 1, U.end()), vv(V.begin() + 1, V.end()), dd(D.begin() + 1, D.end());
  CK(upload(I.d_u, uu, s), "upload grid"); CK(upload(I.d_v, vv, s), "upload grid");
  CK(upload(I.d_depth, dd, s), "upload grid");
  A.klat = I.d_klat.template as<int>(); A.klon = I.d_klon.template as<int>(); A.wlat = I.d_wlat.template as<R>();
  A.dpsn = I.d_dpsn.template as<R>(); A.della0 = I.d_della0.template as<R>(); A.drgm = I.d_drgm.template as<R>();
  A.indep = I.d_indep.template as<int>(); A.indep_g = I.d_indep_g.template as<int>();
  A.ddphi = I.d_ddphi.template as<R>(); A.ddlam = I.d_ddlam.template as<R>();
  A.duphi = I.d_duphi.template as<R>(); A.dulam = I.d_dulam.template as<R>();
  A.dvphi = I.d_dvphi.template as<R>(); A.dvlam = I.d_dvlam.template as<R>();
  A.u = I.d_u.template as<R>(); A.v = I.d_v.template as<R>();
  A.TCGOND = I.tcgond.template as<R>(); A.TSIHKD = I.tsihkd.template as<R>(); A.TFAK = I.tfak.template as<R>();
  A.GOM = I.gom.template as<R>(); A.FR = I.fr.template as<R>();
  for (int k = 0; k < KL; ++k) { A.sinth[k] = t.SINTH[k]; A.costh[k] = t.COSTH[k]; }
  // CHECK_CFL (:1917-2138) from the extrema of the recomputed coefficients
  CK(I.cflext.ensure(2 * CFL_NCLASS * sizeof(long long)), "alloc");
  CK(launch_cfl_extrema<R>(A, I.cflext.template as<long long>(), ctx->nsm, s), "cfl kernel");
  long long ext[2 * CFL_NCLASS];
  CK(cudaMemcpyAsync(ext, I.cflext.p, sizeof(ext), cudaMemcpyDeviceToHost, s), "cfl copy");
  CK(cudaStreamSynchronize(s), "cfl sync");
  auto mx = [&](int q) { return (R)cfl_decode(ext[2 * q], sizeof(R)); };
  auto mn = [&](int q) { return (R)cfl_decode(ext[2 * q + 1], sizeof(R)); };
  const bool cur = c.refraction_c_run;
  const bool has_theta = c.spherical_run || cur || (c.shallow_run && c.refraction_d_run);
  R lat11max = cur ? std::max(mx(CFL_LAT11), mx(CFL_LAT21)) : mx(CFL_LAT11);
  R lat11min = cur ? std::min(mn(CFL_LAT11), mn(CFL_LAT21)) : mn(CFL_LAT11);
  R lat12max = R(0.1), lat12min = R(0.1);
  if (c.reduced_grid) {
    lat12max = cur ? std::max(mx(CFL_LAT12), mx(CFL_LAT22)) : mx(CFL_LAT12);
    lat12min = cur ? std::min(mn(CFL_LAT12), mn(CFL_LAT22)) : mn(CFL_LAT12);
  }
  R lon11max = mx(CFL_LON1);
  R lon12max = cur ? mx(CFL_LON2) : R(0.1), lon12min = cur ? mn(CFL_LON2) : R(0.1);
  R th1max = has_theta ? mx(CFL_TH1) : R(0.1), th1min = has_theta ? mn(CFL_TH1) : R(0.1);
  R th2max = has_theta ? mx(CFL_TH2) : R(0.1), th2min = has_theta ? mn(CFL_TH2) : R(0.1);
  R sg1max = cur ? mx(CFL_SG1) : R(0.1), sg1min = cur ? mn(CFL_SG1) : R(0.1);
  R sg2max = cur ? mx(CFL_SG2) : R(0.1), sg2min = cur ? mn(CFL_SG2) : R(0.1);
  R summax = R(1.) - mn(CFL_SUM), summin = R(1.) - mx(CFL_SUM);
  R cmax = std::max({lat11max, lat12max, lon11max, lon12max, th1max, th2max, sg1max, sg2max, summax});
  // the minimum follows CHECK_CFL's own expression (propagation:2013-2016),
  // which lists COEF_LON_1_2_MIN twice and not COEF_LON_1_1_MIN
  R cmin = std::min({lat11min, lat12min, lon12min, lon12min, th1min, th2min, sg1min, sg2min, summin});
  ctx->cfl_min = cmin;
  if (cmin < R(0.)) {
    ctx->total_cfl = cmin;
    if (total_cfl) *total_cfl = (float)cmin;
    return fail(ctx, WAMGPU_E_CFL, "negative propagation coefficient (CHECK_CFL): reduce IDELPRO");
  }
  R tc = cmax;
  int cnt = 1;
  if (tc > R(0.999)) { cnt = (int)std::ceil(tc); tc = tc / R(cnt); }
  A.counter = cnt; A.rcounter = R(cnt);
  ctx->counter = cnt; ctx->total_cfl = tc;
  if (total_cfl) *total_cfl = (float)tc;
  if (counter) *counter = cnt;
  // per-point source inputs for the host entry points
  I.has_enh = false;
  ctx->prepared = true;
  return WAMGPU_OK;
}

template <typename R> int set_grid_t(wamgpu_ctx* ctx, Impl<R>& I) {
  const int n = ctx->nsea;
  I.dco.assign(n + 1, R(0)); I.dpsn.assign((size_t)2 * n, R(1.));
  if (ctx->cfg.spherical_run) {  // wam_initial_module.f90:204-214
    for (int i = 0; i < n; ++i) I.dco[i + 1] = R(1.) / R(ctx->cosph[ctx->kfromij[i] - 1]);
    for (int i = 0; i < n; ++i)
      for (int ic = 0; ic < 2; ++ic) {
        int nb = ctx->klat[i + n * ic];
        if (nb != 0) I.dpsn[i + (size_t)n * ic] = I.dco[i + 1] / I.dco[nb];
      }
  }
  return WAMGPU_OK;
}

// MAKE_SHALLOW_SNL (:975-1048)
template <typename R> int prepare_source_t(wamgpu_ctx* ctx, Impl<R>& I) {
  const Config& c = ctx->cfg;
  // ST6: WAVNU2 depends on the depth only, so its rows are formed once here
  ctx->wncg_valid = false;
  if (c.iphys == 2 && ctx->prepared) {
    CK(I.wncg.ensure((size_t)ctx->nsea * 2 * c.ml * sizeof(R) + 16), "alloc WN/CG");
    CK(launch_wavnu2<R>(I.dt, I.d_depth.template as<R>(), ctx->nsea, I.wncg.template as<R>(), ctx->stream), "WAVNU2");
    CK(cudaStreamSynchronize(ctx->stream), "WAVNU2");
    ctx->wncg_valid = true;
  }
  I.has_enh = false;
  if (!(c.shallow_run && c.isnonlin != 0)) return WAMGPU_OK;
  const TableSet<R>& t = I.tab;
  const int n = ctx->nsea, mlsthg = t.MLSTHG;
  std::vector<R> enh((size_t)n * mlsthg);
  for (int m = 1; m <= mlsthg; ++m)
    for (int i = 0; i < n; ++i) {
      R d = R(ctx->depth[i]);
      R om = (m <= t.ML) ? Phys<R>::ZPI * t.FR[m - 1] : Phys<R>::ZPI * t.FR[t.ML - 1] * powi(Phys<R>::CO, m - t.ML);
      enh[i + (size_t)n * (m - 1)] = std::min(R(10.), transf(aki(om, d), d));
    }
  CK(upload(I.enh, enh, ctx->stream), "upload ENH");
  I.has_enh = true;
  CK(cudaStreamSynchronize(ctx->stream), "ENH");
  return WAMGPU_OK;
}

template <typename R>
int implsch_dev_t(wamgpu_ctx* ctx, Impl<R>& I, void* fl3, int ld, const void* u10, const void* udir, void* tauw,
                  void* ustar, void* z0, const void* roairn, const void* wstar, cudaStream_t s, const void* fl3_in = nullptr,
                  R* lfout = nullptr) {
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first (INDEP)");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  if (ctx->cfg.shallow_run && ctx->cfg.isnonlin != 0 && !I.has_enh)
    return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_source first (ISNONLIN table)");
  if (!I.status.p) { CK(I.status.ensure(16), "alloc"); CK(cudaMemsetAsync(I.status.p, 0, 16, s), "memset"); }
  if (ctx->cfg.lcflx) CK(I.fluxes.ensure((size_t)7 * ctx->nsea * sizeof(R) + 16), "alloc");
  // the owned sea points only (all of them unless wamgpu_set_owned narrowed the range)
  const int p0 = ctx->own0, p1 = ctx->own1 < 0 ? ctx->nsea : ctx->own1;
  ImplArgs<R> a;
  a.nsea = p1 - p0; a.ld = ld;
  a.fl3 = (R*)fl3 + p0; a.fl3_in = (fl3_in ? (const R*)fl3_in : (const R*)fl3) + p0;
  a.u10 = (const R*)u10 + p0; a.udir = (const R*)udir + p0; a.roairn = (const R*)roairn + p0; a.wstar = (const R*)wstar + p0;
  a.depth = I.d_depth.template as<R>() + p0; a.indep = I.d_indep.template as<int>() + p0;
  a.tauw = (R*)tauw + p0; a.ustar = (R*)ustar + p0; a.z0 = (R*)z0 + p0;
  a.fluxes = ctx->cfg.lcflx ? I.fluxes.template as<R>() + p0 : nullptr;
  a.flx_ld = ctx->nsea;
  a.enh = I.has_enh ? I.enh.template as<R>() + p0 : nullptr; a.enh_ld = ctx->nsea;
  a.wncg = ctx->wncg_valid ? I.wncg.template as<R>() + (size_t)p0 * 2 * ctx->cfg.ml : nullptr;
  a.status = I.status.template as<int>();
  a.lfout = lfout ? lfout + p0 : nullptr;
  if (ctx->diag) {
    a.diag = ctx->diag + p0;
    a.diag_ll = ctx->diag_ll ? ctx->diag_ll + p0 : nullptr;
    a.diag_ld = ctx->diag_ld;
  }
  { TimedLaunch tl(ctx, 1, s); CK(launch_implsch<R>(I.dt, a, ctx->P, s), "implsch launch"); }
  return WAMGPU_OK;
}

template <typename R> int propags_dev_t(wamgpu_ctx* ctx, Impl<R>& I, void* f3v, int ld, void* scratch, cudaStream_t s) {
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  R* f3 = (R*)f3v;
  const size_t bytes = (size_t)ld * ctx->cfg.kl * ctx->cfg.ml * sizeof(R);
  R* sc = (R*)scratch;
  if (!sc) { CK(I.scratch.ensure(bytes), "alloc scratch"); sc = I.scratch.template as<R>(); }
  // ping-pong over COUNTER sub-steps so that the last one writes f3
  const int cnt = ctx->counter;
  R* src = f3; R* dst = sc;
  if (cnt % 2 == 1) { CK(cudaMemcpyAsync(sc, f3, bytes, cudaMemcpyDeviceToDevice, s), "copy F1"); src = sc; dst = f3; }
  for (int it = 0; it < cnt; ++it) {
    { TimedLaunch tl(ctx, 0, s); CK(launch_propags<R>(I.pa, src, ld, dst, ld, s), "propags launch"); }
    std::swap(src, dst);
  }
  return WAMGPU_OK;
}

// Address of the fixed PROPAGS scratch on the context's device, looked up
// once per device with that device current (first call) and kept for the
// process.
constexpr int kMaxStaticDevices = 64;
std::mutex g_static_mu;
void* g_static_addr[kMaxStaticDevices] = {};

int static_scratch(wamgpu_ctx* ctx, void** out) {
  const int dev = ctx->cfg.device;
  if (dev < 0 || dev >= kMaxStaticDevices) return fail(ctx, WAMGPU_E_ARG, "device ordinal beyond the static scratch table");
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_addr[dev]) {
    int prev = -1;
    CK(cudaGetDevice(&prev), "cudaGetDevice");
    if (prev != dev) CK(cudaSetDevice(dev), "cudaSetDevice");
    void* p = nullptr;
    const cudaError_t e = static_scratch_address(&p);
    if (prev != dev) cudaSetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress (static PROPAGS scratch)");
    if (!p) return fail(ctx, WAMGPU_E_CUDA, "static PROPAGS scratch has no device address");
    g_static_addr[dev] = p;
  }
  *out = g_static_addr[dev];
  return WAMGPU_OK;
}

// PROPAGS with the F1 ping-pong spectrum in the fixed device array: no
// allocation, no clearing (each scratch element read was written earlier in
// the call), sizes above the array rejected before anything is queued.
// One PROPAGS sub-step (IDELPRO/COUNTER seconds) from src to dst over the
// owned sea points; halo points of dst are left as they were.
template <typename R> int propags_substep_t(wamgpu_ctx* ctx, Impl<R>& I, const void* src, void* dst, int ld, cudaStream_t s) {
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  if (src == dst) return fail(ctx, WAMGPU_E_ARG, "a sub-step needs distinct source and destination spectra");
  { TimedLaunch tl(ctx, 0, s); CK(launch_propags<R>(I.pa, (const R*)src, ld, (R*)dst, ld, s), "propags launch"); }
  return WAMGPU_OK;
}

// The same over the points [i0, i1) of the owned range only.
template <typename R>
int propags_range_t(wamgpu_ctx* ctx, Impl<R>& I, const void* src, void* dst, int ld, int i0, int i1, cudaStream_t s) {
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  if (src == dst) return fail(ctx, WAMGPU_E_ARG, "a sub-step needs distinct source and destination spectra");
  const int o0 = ctx->own0, o1 = ctx->own1 < 0 ? ctx->nsea : ctx->own1;
  if (i0 < o0 || i1 > o1 || i0 > i1) return fail(ctx, WAMGPU_E_ARG, "point range outside the owned range");
  PropArgs<R> A = I.pa;
  A.i0 = i0; A.i1 = i1;
  { TimedLaunch tl(ctx, 0, s); CK(launch_propags<R>(A, (const R*)src, ld, (R*)dst, ld, s), "propags launch"); }
  return WAMGPU_OK;
}

template <typename R> int set_counter_t(wamgpu_ctx* ctx, Impl<R>& I, int counter) {
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first");
  if (counter < ctx->counter)
    return fail(ctx, WAMGPU_E_ARG, "COUNTER below this grid's own CHECK_CFL value (" + std::to_string(ctx->counter) + ")");
  ctx->total_cfl = ctx->total_cfl * ctx->counter / counter;
  ctx->counter = counter;
  I.pa.counter = counter; I.pa.rcounter = R(counter);
  return WAMGPU_OK;
}

// ---- derivatives (ST4): tangent-linear and adjoint ----------------------------

// The source tables as the point-per-thread derivative code sees them.
template <typename R> adj::ATabs<R> atabs_of(const DevTables<R>& d) {
  adj::ATabs<R> A;
  const SmallLayout& L = d.lay;
  A.KL = d.KL; A.ML = d.ML; A.NDEPTH = d.NDEPTH; A.MFRSTLW = d.MFRSTLW; A.MLSTHG = d.MLSTHG; A.KFRH = d.KFRH;
  A.NSDSNTH = d.NSDSNTH; A.shallow = d.shallow; A.isnonlin = d.isnonlin;
  A.DELTH = d.DELTH; A.INV_LOG_CO = d.INV_LOG_CO; A.MO_TAIL = d.MO_TAIL; A.MM1_TAIL = d.MM1_TAIL; A.DELU = d.DELU;
  A.DAL1 = d.DAL1; A.DAL2 = d.DAL2; A.X0TAUHF = d.X0TAUHF; A.BETAMAX = d.BETAMAX; A.ZALP = d.ZALP; A.ALPHA = d.ALPHA;
  A.TAUWSHELTER = d.TAUWSHELTER; A.DELT = d.DELT;
  const R* r = d.small;
  A.FR = r + L.FR; A.DFIM = r + L.DFIM; A.DFIMOFR = r + L.DFIMOFR; A.FR5 = r + L.FR5; A.FRM5 = r + L.FRM5;
  A.RHOWG = r + L.RHOWG_DFIM; A.TH = r + L.TH; A.COSTH = r + L.COSTH; A.SINTH = r + L.SINTH; A.DELFL = r + L.DELFL;
  A.AF11 = r + L.AF11; A.RNL = r + L.RNLCOEF; A.SATW = r + L.SATW; A.WTAUHF = r + L.WTAUHF; A.SWELLFT = r + L.SWELLFT;
  A.TFAK = d.TFAK; A.TCGOND = d.TCGOND; A.FLMINFR = d.FLMINFR;
  const int* q = d.ismall;
  A.K1W = q + L.K1W; A.K2W = q + L.K2W; A.K11W = q + L.K11W; A.K21W = q + L.K21W; A.INL = q + L.INLCOEF;
  A.IKP = q + L.IKP; A.IKP1 = q + L.IKP1; A.IKM = q + L.IKM; A.IKM1 = q + L.IKM1; A.INDSAT = q + L.INDSAT;
  return A;
}

template <typename R>
int deriv_setup(wamgpu_ctx* ctx, Impl<R>& I, int ld, bool tl, DerivArgs<R>& a) {
  if (tl && ctx->cfg.iphys != 1)
    return fail(ctx, WAMGPU_E_ARG, "the IMPLSCH tangent-linear is implemented for ST4 (IPHYS=1)");
  if (ctx->cfg.iphys == 2) {
    // the ST6 adjoint keeps its LFACTOR record and row adjoints in the tape rows
    const int ml = ctx->cfg.ml, nk10 = I.dt.NK10;
    if (14 * ml - 16 < std::max(6 * ml, 2 * nk10 + ml))
      return fail(ctx, WAMGPU_E_ARG, "ST6 adjoint: frequency grid too short for the 10 Hz extension's tape rows");
  }
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first (INDEP)");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  if (ctx->own0 != 0 || (ctx->own1 >= 0 && ctx->own1 != ctx->nsea))
    return fail(ctx, WAMGPU_E_ARG, "derivatives cover the whole grid of a context (no owned range)");
  if (ctx->cfg.shallow_run && ctx->cfg.isnonlin != 0 && !I.has_enh)
    return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_source first (ISNONLIN table)");
  if (ctx->cfg.kl > 64) return fail(ctx, WAMGPU_E_ARG, "IMPLSCH derivatives support at most 64 directions");
  {
    // the adjoint gathers the transposed saturation window per direction
    // column: INDICESSAT(K, J) must be the rotation K + J - NSDSNTH (ST4)
    const TableSet<R>& t = I.tab;
    const int KL = t.KL, ns = t.NSDSNTH;
    for (int j = 0; ctx->cfg.iphys == 1 && j < 2 * ns + 1; ++j)
      for (int k = 0; k < KL; ++k)
        if (t.INDICESSAT[k + KL * j] - 1 != ((k + j - ns) % KL + KL) % KL)
          return fail(ctx, WAMGPU_E_ARG, "saturation window is not a rotation of the directions");
  }
  const size_t n = (size_t)ctx->nsea;
  if (tl) {
    CK(I.dwork.ensure(n * deriv_work_bytes<R>(ctx->cfg.kl, ctx->cfg.ml) + 256), "alloc derivative work");
    CK(I.dmasks.ensure(n * 2 * ctx->cfg.kl * ctx->cfg.ml + 256), "alloc derivative work");
  }
  std::memset(&a, 0, sizeof(a));
  a.A = atabs_of(I.dt);
  a.nsea = ctx->nsea; a.ld = ld;
  a.depth = I.d_depth.template as<R>(); a.indep = I.d_indep.template as<int>();
  a.enh = I.has_enh ? I.enh.template as<R>() : nullptr; a.enh_ld = ctx->nsea;
  a.work = I.dwork.p; a.masks = I.dmasks.template as<uint8_t>();
  return WAMGPU_OK;
}

template <typename R>
int implsch_adj_t(wamgpu_ctx* ctx, Impl<R>& I, const void* fl3_in, int ld, const void* tauw_in, const void* u10,
                  const void* udir, const void* roairn, const void* wstar, void* lam_fl3, void* lam_tauw, void* lam_u10,
                  cudaStream_t s, void* lam_out = nullptr, const R* lfin = nullptr) {
  DerivArgs<R> a;
  int rc = deriv_setup<R>(ctx, I, ld, false, a);
  if (rc) return rc;
  a.lam_out = (R*)lam_out;
  a.lfin = lfin;
  a.fl3_in = (const R*)fl3_in; a.tauw_in = (const R*)tauw_in; a.u10 = (const R*)u10; a.udir = (const R*)udir;
  a.roairn = (const R*)roairn; a.wstar = (const R*)wstar;
  a.lam_fl3 = (R*)lam_fl3; a.lam_tauw = (R*)lam_tauw; a.lam_u10 = (R*)lam_u10;
  { TimedLaunch tl(ctx, 1, s); CK(launch_implsch_adj<R>(I.dt, a, s), "implsch adjoint launch"); }
  return WAMGPU_OK;
}

template <typename R>
int implsch_tl_t(wamgpu_ctx* ctx, Impl<R>& I, const void* fl3_in, const void* dfl3_in, int ld, const void* tauw_in,
                 const void* dtauw_in, const void* u10, const void* du10, const void* udir, const void* roairn,
                 const void* wstar, void* fl3_out, void* dfl3_out, void* tauw_out, void* dtauw_out, cudaStream_t s) {
  DerivArgs<R> a;
  int rc = deriv_setup<R>(ctx, I, ld, true, a);
  if (rc) return rc;
  a.fl3_in = (const R*)fl3_in; a.dfl3_in = (const R*)dfl3_in; a.tauw_in = (const R*)tauw_in;
  a.dtauw_in = (const R*)dtauw_in; a.u10 = (const R*)u10; a.du10 = (const R*)du10; a.udir = (const R*)udir;
  a.roairn = (const R*)roairn; a.wstar = (const R*)wstar;
  a.fl3_out = (R*)fl3_out; a.dfl3_out = (R*)dfl3_out; a.tauw_out = (R*)tauw_out; a.dtauw_out = (R*)dtauw_out;
  CK(launch_implsch_tl<R>(a, s), "implsch tangent-linear launch");
  return WAMGPU_OK;
}

// Transpose of PROPAGS: the COUNTER sub-steps in reverse order, ping-pong
// between lam and scratch (zeroed before each sub-step).
template <typename R> int propags_adj_t(wamgpu_ctx* ctx, Impl<R>& I, void* lam, int ld, void* scratch, cudaStream_t s) {
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  const size_t bytes = (size_t)ld * ctx->cfg.kl * ctx->cfg.ml * sizeof(R);
  R* sc = (R*)scratch;
  if (!sc) { CK(I.scratch.ensure(bytes), "alloc scratch"); sc = I.scratch.template as<R>(); }
  R* src = (R*)lam; R* dst = sc;
  for (int it = 0; it < ctx->counter; ++it) {
    CK(cudaMemsetAsync(dst, 0, bytes, s), "zero adjoint");
    { TimedLaunch tl(ctx, 0, s); CK(launch_propags_adj<R>(I.pa, src, ld, dst, ld, s), "propags adjoint launch"); }
    std::swap(src, dst);
  }
  if (src != (R*)lam) CK(cudaMemcpyAsync(lam, src, bytes, cudaMemcpyDeviceToDevice, s), "copy adjoint");
  return WAMGPU_OK;
}

// ---- checkpointed assimilation windows ------------------------------------------

// Slot q of the checkpoint store: the spectrum entering IMPLSCH (pitch
// ckpt_ld), then TAUW before IMPLSCH, U10 and, for ST6, the RTAU of
// LFACTOR's last round (NSEA values each), so that the adjoint repeats only
// that round.
template <typename R> R* ckpt_slot(const wamgpu_ctx* ctx, Impl<R>& I, int q) {
  const size_t per = (size_t)I.ckpt_ld * ctx->cfg.kl * ctx->cfg.ml + 3 * (size_t)ctx->nsea;
  return I.ckpt.template as<R>() + per * q;
}

template <typename R> int checkpoint_reserve_t(wamgpu_ctx* ctx, Impl<R>& I, int n, int ld) {
  if (n < 0) return fail(ctx, WAMGPU_E_ARG, "negative number of checkpoints");
  if (n == 0) { I.ckpt = DevBuf(); I.nckpt = 0; I.ckpt_ld = 0; return WAMGPU_OK; }
  if (!ctx->have_grid) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_set_grid first");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  const size_t per = (size_t)ld * ctx->cfg.kl * ctx->cfg.ml + 3 * (size_t)ctx->nsea;
  CK(I.ckpt.ensure(per * n * sizeof(R)), "alloc checkpoints");
  I.nckpt = n; I.ckpt_ld = ld;
  return WAMGPU_OK;
}

template <typename R> int ckpt_check(wamgpu_ctx* ctx, Impl<R>& I, int slot, int ld, int nprop) {
  if (slot < 0 || slot >= I.nckpt) return fail(ctx, WAMGPU_E_ARG, "checkpoint slot outside wamgpu_checkpoint_reserve's range");
  if (ld != I.ckpt_ld) return fail(ctx, WAMGPU_E_ARG, "ld differs from the ld given to wamgpu_checkpoint_reserve");
  if (nprop < 0) return fail(ctx, WAMGPU_E_ARG, "nprop < 0");
  return WAMGPU_OK;
}

// wamgpu_step_dev that also stores checkpoint `slot`.
template <typename R>
int step_ckpt_dev_t(wamgpu_ctx* ctx, Impl<R>& I, int slot, void* f3v, int ld, void* scratch, int nprop, const void* u10,
                    const void* udir, void* tauw, void* ustar, void* z0, const void* roairn, const void* wstar,
                    cudaStream_t s) {
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first");
  int rc = ckpt_check(ctx, I, slot, ld, nprop);
  if (rc) return rc;
  R* f3 = (R*)f3v;
  const size_t nb = (size_t)ctx->cfg.kl * ctx->cfg.ml, bytes = (size_t)ld * nb * sizeof(R);
  R* sc = (R*)scratch;
  if (!sc) { CK(I.scratch.ensure(bytes), "alloc scratch"); sc = I.scratch.template as<R>(); }
  R* src = f3; R* dst = sc;
  for (int it = 0; it < nprop * ctx->counter; ++it) {
    { TimedLaunch tl(ctx, 0, s); CK(launch_propags<R>(I.pa, src, ld, dst, ld, s), "propags launch"); }
    std::swap(src, dst);
  }
  R* c = ckpt_slot(ctx, I, slot);
  const size_t n = (size_t)ctx->nsea;
  CK(cudaMemcpyAsync(c, src, bytes, cudaMemcpyDeviceToDevice, s), "checkpoint spectrum");
  CK(cudaMemcpyAsync(c + (size_t)ld * nb, tauw, n * sizeof(R), cudaMemcpyDeviceToDevice, s), "checkpoint TAUW");
  CK(cudaMemcpyAsync(c + (size_t)ld * nb + n, u10, n * sizeof(R), cudaMemcpyDeviceToDevice, s), "checkpoint U10");
  return implsch_dev_t<R>(ctx, I, f3, ld, u10, udir, tauw, ustar, z0, roairn, wstar, s, src,
                          ctx->cfg.iphys == 2 ? c + (size_t)ld * nb + 2 * n : nullptr);
}

// The adjoint of the step stored in `slot`: IMPLSCH's adjoint at the
// checkpoint, then the transposes of the step's nprop PROPAGS calls.
template <typename R>
int step_adj_dev_t(wamgpu_ctx* ctx, Impl<R>& I, int slot, int nprop, void* lam_fl3, int ld, void* lam_tauw, void* lam_u10,
                   const void* udir, const void* roairn, const void* wstar, void* scratch, cudaStream_t s) {
  int rc = ckpt_check(ctx, I, slot, ld, nprop);
  if (rc) return rc;
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first");
  const R* c = ckpt_slot(ctx, I, slot);
  const size_t nb = (size_t)ctx->cfg.kl * ctx->cfg.ml, bytes = (size_t)ld * nb * sizeof(R);
  R* lam = (R*)lam_fl3;
  R* sc = (R*)scratch;
  if (!sc) { CK(I.scratch.ensure(bytes), "alloc scratch"); sc = I.scratch.template as<R>(); }
  // the sub-steps ping-pong between lam and scratch; the IMPLSCH adjoint
  // writes where the first one must start so that the last one ends in lam
  const int nsub = nprop * ctx->counter;
  R* src = (nsub % 2) ? sc : lam;
  rc = implsch_adj_t<R>(ctx, I, c, ld, c + (size_t)ld * nb, c + (size_t)ld * nb + ctx->nsea, udir, roairn, wstar, lam,
                        lam_tauw, lam_u10, s, src == lam ? nullptr : src,
                        ctx->cfg.iphys == 2 ? c + (size_t)ld * nb + 2 * (size_t)ctx->nsea : nullptr);
  if (rc) return rc;
  R* dst = src == lam ? sc : lam;
  for (int it = 0; it < nsub; ++it) {
    CK(cudaMemsetAsync(dst, 0, bytes, s), "zero adjoint");
    { TimedLaunch tl(ctx, 0, s); CK(launch_propags_adj<R>(I.pa, src, ld, dst, ld, s), "propags adjoint launch"); }
    std::swap(src, dst);
  }
  return WAMGPU_OK;
}

template <typename R> int propags_dev_static_t(wamgpu_ctx* ctx, Impl<R>& I, void* f3v, int ld, cudaStream_t s) {
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  // With an owned range the sub-steps write only the owned points of the
  // scratch, and the next sub-step would read halo points of it that this
  // call never wrote (whatever an earlier call left in the shared array).
  if (ctx->own0 != 0 || (ctx->own1 >= 0 && ctx->own1 != ctx->nsea))
    return fail(ctx, WAMGPU_E_ARG,
                "wamgpu_propags_dev_static covers the whole grid; with an owned range (wamgpu_set_owned) use "
                "wamgpu_propags_substep_dev and refresh the halo between sub-steps");
  const size_t bytes = (size_t)ld * ctx->cfg.kl * ctx->cfg.ml * sizeof(R);
  if (bytes > (size_t)WAMGPU_STATIC_SCRATCH_BYTES)
    return fail(ctx, WAMGPU_E_ARG, "spectrum of " + std::to_string(bytes) + " bytes exceeds the static PROPAGS scratch of " +
                                       std::to_string((size_t)WAMGPU_STATIC_SCRATCH_BYTES) +
                                       " bytes; use wamgpu_propags_dev with a scratch spectrum");
  void* base = nullptr;
  const int rc = static_scratch(ctx, &base);
  if (rc) return rc;
  R* f3 = (R*)f3v;
  R* sc = (R*)base;
  const int cnt = ctx->counter;
  R* src = f3; R* dst = sc;
  if (cnt % 2 == 1) { CK(cudaMemcpyAsync(sc, f3, bytes, cudaMemcpyDeviceToDevice, s), "copy F1"); src = sc; dst = f3; }
  for (int it = 0; it < cnt; ++it) {
    CK(launch_propags<R>(I.pa, src, ld, dst, ld, s), "propags launch");
    std::swap(src, dst);
  }
  return WAMGPU_OK;
}

// One pass of WAMODEL's PROP/PHYSICS loop body (wamodel.f90:286-360): nprop
// PROPAGS calls (each COUNTER sub-steps) followed by one IMPLSCH.  All
// sub-steps ping-pong between f3 and scratch and IMPLSCH reads whichever
// buffer the last one wrote, writing its result into f3: no device copies.
template <typename R>
int step_dev_t(wamgpu_ctx* ctx, Impl<R>& I, void* f3v, int ld, void* scratch, int nprop, const void* u10, const void* udir,
               void* tauw, void* ustar, void* z0, const void* roairn, const void* wstar, cudaStream_t s) {
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  if (nprop < 0) return fail(ctx, WAMGPU_E_ARG, "nprop < 0");
  R* f3 = (R*)f3v;
  const size_t bytes = (size_t)ld * ctx->cfg.kl * ctx->cfg.ml * sizeof(R);
  R* sc = (R*)scratch;
  if (!sc) { CK(I.scratch.ensure(bytes), "alloc scratch"); sc = I.scratch.template as<R>(); }
  R* src = f3; R* dst = sc;
  for (int it = 0; it < nprop * ctx->counter; ++it) {
    { TimedLaunch tl(ctx, 0, s); CK(launch_propags<R>(I.pa, src, ld, dst, ld, s), "propags launch"); }
    std::swap(src, dst);
  }
  return implsch_dev_t<R>(ctx, I, f3, ld, u10, udir, tauw, ustar, z0, roairn, wstar, s, src);
}

// COMPUTE_OUTPUT_PARAMETER (wam_output_module.f90:481-640) for the owned
// sea points: the integrated parameters into block[ij + block_ld*(IP-1)].
template <typename R>
int output_params_t(wamgpu_ctx* ctx, Impl<R>& I, const void* fl3, int ld, const void* u10, const void* udir,
                    const void* tauw, void* ustar, void* z0, int from, void* block, int block_ld, cudaStream_t s) {
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first (INDEP, currents)");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  if (block_ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "block_ld < nsea");
  if (!fl3 || !u10 || !udir || !tauw || !ustar || !z0 || !block) return fail(ctx, WAMGPU_E_ARG, "null argument");
  const int p0 = ctx->own0, p1 = ctx->own1 < 0 ? ctx->nsea : ctx->own1;
  const DevTables<R>& d = I.dt;
  OutArgs<R> a;
  a.nsea = p1 - p0; a.ld = ld; a.KL = d.KL; a.ML = d.ML; a.NDEPTH = d.NDEPTH; a.shallow = d.shallow;
  a.from = from ? 1 : 0;
  a.fl3 = (const R*)fl3 + p0;
  a.u10 = (const R*)u10 + p0; a.udir = (const R*)udir + p0; a.tauw = (const R*)tauw + p0;
  a.depth = I.d_depth.template as<R>() + p0;
  a.u = I.d_u.template as<R>() + p0;  // zero unless wamgpu_set_current gave currents
  a.v = I.d_v.template as<R>() + p0;
  a.ustar = (R*)ustar + p0; a.z0 = (R*)z0 + p0;
  a.indep = I.d_indep.template as<int>() + p0;
  a.block = (R*)block + p0; a.block_ld = block_ld;
  const R* r = d.small;
  a.FR = r + d.lay.FR; a.DFIM = r + d.lay.DFIM; a.DFIMOFR = r + d.lay.DFIMOFR;
  a.SINTH = r + d.lay.SINTH; a.COSTH = r + d.lay.COSTH;
  const R* ot = I.outtab.template as<R>();
  a.DFIM_FR = ot; a.DFIM_FR2 = ot + d.ML; a.MSSFD = ot + 2 * d.ML;
  a.TFAK = d.TFAK;
  a.MO_TAIL = d.MO_TAIL; a.MM1_TAIL = d.MM1_TAIL;
  a.MP1_TAIL = R(I.tab.MP1_TAIL); a.MP2_TAIL = R(I.tab.MP2_TAIL);
  a.A = atabs_of(d);
  a.ustar_max = nullptr;
  CK(I.ustar_max.ensure(16), "alloc");
  // parameters that are not computed stay 0
  for (int p = 0; p < WAMGPU_OUT_NPARAM; ++p)
    CK(cudaMemsetAsync((R*)block + p0 + (size_t)block_ld * p, 0, (size_t)(p1 - p0) * sizeof(R), s), "memset block");
  CK(launch_output<R>(a, I.ustar_max.template as<unsigned long long>(), s), "output launch");
  return WAMGPU_OK;
}

// SWELL_SEPARATION (wam_swell_module.f90:106-350) without the partitioning:
// parameters 17-23 (wind sea) and 25-31 (swell) of the output block.
template <typename R>
int output_swell_t(wamgpu_ctx* ctx, Impl<R>& I, const void* fl3, int ld, const void* udir, const void* ustar, int from,
                   void* block, int block_ld, cudaStream_t s) {
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  if (block_ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "block_ld < nsea");
  if (!fl3 || !udir || !ustar || !block) return fail(ctx, WAMGPU_E_ARG, "null argument");
  const int p0 = ctx->own0, p1 = ctx->own1 < 0 ? ctx->nsea : ctx->own1;
  const DevTables<R>& d = I.dt;
  OutArgs<R> a;
  a.nsea = p1 - p0; a.ld = ld; a.KL = d.KL; a.ML = d.ML; a.NDEPTH = d.NDEPTH; a.shallow = d.shallow;
  a.from = from ? 1 : 0;
  a.fl3 = (const R*)fl3 + p0;
  a.udir = (const R*)udir + p0;
  a.ustar = const_cast<R*>((const R*)ustar) + p0;
  a.block = (R*)block + p0; a.block_ld = block_ld;
  const R* r = d.small;
  a.FR = r + d.lay.FR; a.DFIM = r + d.lay.DFIM; a.DFIMOFR = r + d.lay.DFIMOFR;
  a.SINTH = r + d.lay.SINTH; a.COSTH = r + d.lay.COSTH; a.TH = r + d.lay.TH;
  const R* ot = I.outtab.template as<R>();
  a.DFIM_FR = ot; a.DFIM_FR2 = ot + d.ML; a.MSSFD = ot + 2 * d.ML; a.C = ot + 3 * d.ML;
  a.MO_TAIL = d.MO_TAIL; a.MM1_TAIL = d.MM1_TAIL;
  a.MP1_TAIL = R(I.tab.MP1_TAIL); a.MP2_TAIL = R(I.tab.MP2_TAIL);
  CK(launch_swell<R>(a, s), "swell launch");
  return WAMGPU_OK;
}

// PUT_ICE (wam_ice_module.f90:312-324) / PUT_DRY (wam_topo_module.f90:557-569)
// on device data of nrows rows (a spectrum: KL*ML rows; a parameter block:
// its parameters), skipping listed points outside the owned range as the
// reference skips those outside NIJS..NIJL.
template <typename R>
int put_points_t(wamgpu_ctx* ctx, Impl<R>& I, void* data, int ld, int nrows, const int* points, int n, double value,
                 cudaStream_t s) {
  (void)I;
  if (!ctx->have_grid) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_set_grid first");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  if (nrows < 0 || n < 0 || (n > 0 && (!points || !data))) return fail(ctx, WAMGPU_E_ARG, "bad point list");
  const int lo = ctx->own0 + 1, hi = ctx->own1 < 0 ? ctx->nsea : ctx->own1;
  CK(launch_put_points<R>((R*)data, (size_t)ld, nrows, points, n, lo, hi, R(value), s), "put points launch");
  return WAMGPU_OK;
}

// INITIALIZE of INTERPOLATION_TO_GRID (wam_wind_module.f90:1296-1375): per
// sea point the input-grid cell (I1, I2, K1, K2) and the weights DI, DK, in
// the reference's integer 1/100 arc-second units and REAL arithmetic.
template <typename R>
int set_wind_grid_t(wamgpu_ctx* ctx, Impl<R>& I, int nx_in, int ny_in, int west_in, int south_in, int dx_in, int dy_in,
                    int per, int equal, int amowep, int amosop, int xdella, const int* zdello, const int* ifromij) {
  if (!ctx->have_grid) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_set_grid first");
  if (nx_in < 1 || ny_in < 1 || !ifromij || (!equal && (!zdello || dx_in == 0 || dy_in == 0)))
    return fail(ctx, WAMGPU_E_ARG, "wind grid: bad dimensions or missing tables");
  const int n = ctx->nsea;
  const long long M_S_PER = 360LL * 360000LL;
  std::vector<int> tab(4 * (size_t)n);
  std::vector<R> w(2 * (size_t)n, R(0));
  for (int ij = 0; ij < n; ++ij) {
    const int kf = ctx->kfromij[ij], ifr = ifromij[ij];
    int i1, i2, k1, k2;
    if (equal) {
      i1 = i2 = ifr; k1 = k2 = kf;
    } else {
      if (kf < 1 || kf > ctx->ny) return fail(ctx, WAMGPU_E_ARG, "KFROMIJ outside the grid rows");
      long long li = (long long)amowep + (long long)(ifr - 1) * zdello[kf - 1] - west_in;
      li = (li + 2 * M_S_PER) % M_S_PER;
      R di = R((int)li) / R(dx_in);
      const long long lk = (long long)amosop + (long long)(kf - 1) * xdella - south_in;
      R dk = R((int)lk) / R(dy_in);
      i1 = (int)di + 1; k1 = (int)dk + 1;
      k2 = std::min(ny_in, k1 + 1);
      i2 = i1 + 1;
      di = di - R(i1) + R(1.);
      dk = dk - R(k1) + R(1.);
      if (per) { if (i1 == nx_in) i2 = 1; if (i1 == 0) i1 = nx_in; }
      else if (i1 == nx_in) i2 = nx_in;
      w[ij] = di; w[ij + n] = dk;
    }
    if (i1 < 1 || i1 > nx_in || k1 < 1 || k1 > ny_in)
      return fail(ctx, WAMGPU_E_ARG, "sea point " + std::to_string(ij + 1) + " lies outside the wind input grid");
    tab[ij] = i1; tab[ij + n] = i2; tab[ij + 2 * (size_t)n] = k1; tab[ij + 3 * (size_t)n] = k2;
  }
  CK(upload(I.wind_tab, tab, ctx->stream), "upload wind tables");
  CK(upload(I.wind_w, w, ctx->stream), "upload wind tables");
  CK(cudaStreamSynchronize(ctx->stream), "wind tables");
  ctx->wind_nx = nx_in; ctx->wind_ny = ny_in; ctx->wind_equal = equal ? 1 : 0;
  return WAMGPU_OK;
}

template <typename R>
int wind_dev_t(wamgpu_ctx* ctx, Impl<R>& I, const void* u_in, const void* v_in, int code_in, void* u10, void* udir,
               cudaStream_t s) {
  if (ctx->wind_nx <= 0) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_set_wind_grid first");
  if (code_in < 1 || code_in > 3) return fail(ctx, WAMGPU_E_ARG, "wind code must be 1 (USTAR), 2 (stress) or 3 (U10)");
  if (!u_in || !v_in || !u10 || !udir) return fail(ctx, WAMGPU_E_ARG, "null argument");
  CK(launch_wind<R>((const R*)u_in, (const R*)v_in, ctx->wind_nx, ctx->nsea, I.wind_tab.template as<int>(),
                    I.wind_w.template as<R>(), ctx->wind_equal, code_in, (R*)u10, (R*)udir, s), "wind launch");
  return WAMGPU_OK;
}

// ---- restart files (wam_restart_module.f90) ---------------------------------
// The reference writes them as Fortran sequential unformatted records: a
// 4-byte length, the payload, the length again (the layout of gfortran and
// ifort for records below 2 GiB).  Record 1 holds NSEA and the dates CDTPRO,
// CDTSOU, CDA, CDTA, CDCA (CHARACTER(14)); then U10, UDIR, TAUW, FL3 and,
// when their dates are not blank, DEPTH and U with V (one record).  Without
// the spatial decomposition (L_DECOMP false) file position p holds model
// point IJ2NEWIJ(p) (:198-211, :540-559).
constexpr size_t kRestartChunkFloats = size_t(8) << 20;  // 32 MiB staging per copy

bool blank14(const char* c) {
  for (int i = 0; i < 14; ++i) if (c[i] != ' ' && c[i] != 0) return false;
  return true;
}

template <typename R>
int restart_setup(wamgpu_ctx* ctx, Impl<R>& I, int ld, const int* ij2newij, const int** perm_dev) {
  if (!ctx->have_grid) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_set_grid first");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "ld < nsea");
  if (ctx->own0 != 0 || (ctx->own1 >= 0 && ctx->own1 != ctx->nsea))
    return fail(ctx, WAMGPU_E_ARG, "restart files hold the whole grid; this context has an owned range");
  const size_t rec = (size_t)ctx->nsea * ctx->cfg.kl * ctx->cfg.ml * 4;
  if (rec > (size_t)INT_MAX)
    return fail(ctx, WAMGPU_E_ARG, "spectrum record of " + std::to_string(rec) + " bytes exceeds the 2 GiB of one "
                                   "unformatted record");
  *perm_dev = nullptr;
  if (ij2newij) {
    std::vector<char> seen(ctx->nsea + 1, 0);
    for (int p = 0; p < ctx->nsea; ++p) {
      const int q = ij2newij[p];
      if (q < 1 || q > ctx->nsea || seen[q]) return fail(ctx, WAMGPU_E_ARG, "IJ2NEWIJ is not a permutation of 1..NSEA");
      seen[q] = 1;
    }
    std::vector<int> v(ij2newij, ij2newij + ctx->nsea);
    CK(upload(I.rst_perm, v, ctx->stream), "upload IJ2NEWIJ");
    *perm_dev = I.rst_perm.template as<int>();
  }
  CK(I.rst_stage.ensure(kRestartChunkFloats * 4), "alloc restart staging");
  return WAMGPU_OK;
}

template <typename R>
int restart_write_t(wamgpu_ctx* ctx, Impl<R>& I, const char* path, const void* fl3, int ld, const void* u10,
                    const void* udir, const void* tauw, const void* depth, const void* cu, const void* cv,
                    const wamgpu_restart_dates* dates, const int* ij2newij) {
  if (!path || !fl3 || !u10 || !udir || !tauw || !dates) return fail(ctx, WAMGPU_E_ARG, "null argument");
  const bool has_d = !blank14(dates->cdta), has_c = !blank14(dates->cdca);
  if ((has_d && !depth) || (has_c && (!cu || !cv)))
    return fail(ctx, WAMGPU_E_ARG, "CDTA / CDCA set without the depth / current fields");
  const int* perm = nullptr;
  int rc = restart_setup(ctx, I, ld, ij2newij, &perm);
  if (rc) return rc;
  const int n = ctx->nsea;
  cudaStream_t s = ctx->stream;
  CK(cudaStreamSynchronize(s), "restart: pending work");
  float* host = nullptr;
  CK(cudaMallocHost(&host, kRestartChunkFloats * 4), "restart: pinned staging");
  std::unique_ptr<float, cudaError_t (*)(void*)> hold(host, cudaFreeHost);
  std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path, "wb"), std::fclose);
  if (!f) return fail(ctx, WAMGPU_E_ARG, std::string("cannot open ") + path + " for writing");
  auto raw = [&](const void* p, size_t bytes) { return std::fwrite(p, 1, bytes, f.get()) == bytes; };
  auto marker = [&](size_t bytes) { const int32_t m = (int32_t)bytes; return raw(&m, 4); };
  // rows of a device array, gathered into file order in chunks
  auto rows = [&](const void* src, size_t sld, int nrows) -> int {
    const int per = (int)std::max<size_t>(1, kRestartChunkFloats / (size_t)n);
    for (int b0 = 0; b0 < nrows; b0 += per) {
      const int nb = std::min(per, nrows - b0);
      CK(launch_restart_gather<R>((const R*)src, sld, n, perm, b0, nb, I.rst_stage.template as<float>(), s),
         "restart gather");
      CK(cudaMemcpyAsync(host, I.rst_stage.p, (size_t)n * nb * 4, cudaMemcpyDeviceToHost, s), "restart D2H");
      CK(cudaStreamSynchronize(s), "restart D2H");
      if (!raw(host, (size_t)n * nb * 4)) return fail(ctx, WAMGPU_E_ARG, std::string("write error on ") + path);
    }
    return WAMGPU_OK;
  };
  auto record = [&](std::initializer_list<std::pair<const void*, std::pair<size_t, int>>> parts) -> int {
    size_t bytes = 0;
    for (auto& q : parts) bytes += (size_t)n * q.second.second * 4;
    if (!marker(bytes)) return fail(ctx, WAMGPU_E_ARG, std::string("write error on ") + path);
    for (auto& q : parts) { const int r = rows(q.first, q.second.first, q.second.second); if (r) return r; }
    if (!marker(bytes)) return fail(ctx, WAMGPU_E_ARG, std::string("write error on ") + path);
    return WAMGPU_OK;
  };
  {
    char head[74];
    const int32_t nn = n;
    std::memcpy(head, &nn, 4);
    std::memcpy(head + 4, dates->cdtpro, 14); std::memcpy(head + 18, dates->cdtsou, 14);
    std::memcpy(head + 32, dates->cda, 14); std::memcpy(head + 46, dates->cdta, 14); std::memcpy(head + 60, dates->cdca, 14);
    if (!marker(74) || !raw(head, 74) || !marker(74)) return fail(ctx, WAMGPU_E_ARG, std::string("write error on ") + path);
  }
  const size_t one = (size_t)n;
  if ((rc = record({{u10, {one, 1}}}))) return rc;
  if ((rc = record({{udir, {one, 1}}}))) return rc;
  if ((rc = record({{tauw, {one, 1}}}))) return rc;
  if ((rc = record({{fl3, {(size_t)ld, ctx->cfg.kl * ctx->cfg.ml}}}))) return rc;
  if (has_d && (rc = record({{depth, {one, 1}}}))) return rc;
  if (has_c && (rc = record({{cu, {one, 1}}, {cv, {one, 1}}}))) return rc;
  if (std::fflush(f.get()) != 0) return fail(ctx, WAMGPU_E_ARG, std::string("write error on ") + path);
  return WAMGPU_OK;
}

template <typename R>
int restart_read_t(wamgpu_ctx* ctx, Impl<R>& I, const char* path, void* fl3, int ld, void* u10, void* udir, void* tauw,
                   void* depth, void* cu, void* cv, wamgpu_restart_dates* dates, const int* ij2newij) {
  if (!path || !fl3 || !u10 || !udir || !tauw) return fail(ctx, WAMGPU_E_ARG, "null argument");
  const int* perm = nullptr;
  int rc = restart_setup(ctx, I, ld, ij2newij, &perm);
  if (rc) return rc;
  const int n = ctx->nsea;
  cudaStream_t s = ctx->stream;
  std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path, "rb"), std::fclose);
  if (!f) return fail(ctx, WAMGPU_E_ARG, std::string("cannot open ") + path);
  float* host = nullptr;
  CK(cudaMallocHost(&host, kRestartChunkFloats * 4), "restart: pinned staging");
  std::unique_ptr<float, cudaError_t (*)(void*)> hold(host, cudaFreeHost);
  auto raw = [&](void* p, size_t bytes) { return std::fread(p, 1, bytes, f.get()) == bytes; };
  auto bad = [&](const std::string& what) { return fail(ctx, WAMGPU_E_ARG, std::string("restart file ") + path + ": " + what); };
  auto marker = [&](size_t want) -> bool { int32_t m = -1; return raw(&m, 4) && (size_t)m == want; };
  auto rows = [&](void* dst, size_t dld, int nrows) -> int {
    const int per = (int)std::max<size_t>(1, kRestartChunkFloats / (size_t)n);
    for (int b0 = 0; b0 < nrows; b0 += per) {
      const int nb = std::min(per, nrows - b0);
      if (!raw(host, (size_t)n * nb * 4)) return bad("short record");
      CK(cudaMemcpyAsync(I.rst_stage.p, host, (size_t)n * nb * 4, cudaMemcpyHostToDevice, s), "restart H2D");
      CK(launch_restart_scatter<R>(I.rst_stage.template as<float>(), n, perm, b0, nb, (R*)dst, dld, s), "restart scatter");
      CK(cudaStreamSynchronize(s), "restart H2D");
    }
    return WAMGPU_OK;
  };
  auto record = [&](std::initializer_list<std::pair<void*, std::pair<size_t, int>>> parts) -> int {
    size_t bytes = 0;
    for (auto& q : parts) bytes += (size_t)n * q.second.second * 4;
    if (!marker(bytes)) return bad("record length differs from the model grid's");
    for (auto& q : parts) {
      if (q.first) { const int r = rows(q.first, q.second.first, q.second.second); if (r) return r; }
      else if (std::fseek(f.get(), (long)((size_t)n * q.second.second * 4), SEEK_CUR) != 0) return bad("short record");
    }
    if (!marker(bytes)) return bad("record length differs from the model grid's");
    return WAMGPU_OK;
  };
  char head[74];
  if (!marker(74) || !raw(head, 74) || !marker(74)) return bad("no header record");
  int32_t nsea_r;
  std::memcpy(&nsea_r, head, 4);
  if (nsea_r != n)
    return bad("NSEA " + std::to_string(nsea_r) + " in the file, " + std::to_string(n) + " in the model grid");
  wamgpu_restart_dates dt;
  std::memcpy(dt.cdtpro, head + 4, 14); std::memcpy(dt.cdtsou, head + 18, 14); std::memcpy(dt.cda, head + 32, 14);
  std::memcpy(dt.cdta, head + 46, 14); std::memcpy(dt.cdca, head + 60, 14);
  if (dates) *dates = dt;
  CK(cudaStreamSynchronize(s), "restart: pending work");
  const size_t one = (size_t)n;
  if ((rc = record({{u10, {one, 1}}}))) return rc;
  if ((rc = record({{udir, {one, 1}}}))) return rc;
  if ((rc = record({{tauw, {one, 1}}}))) return rc;
  if ((rc = record({{fl3, {(size_t)ld, ctx->cfg.kl * ctx->cfg.ml}}}))) return rc;
  if (!blank14(dt.cdta) && (rc = record({{depth, {one, 1}}}))) return rc;
  if (!blank14(dt.cdca) && (rc = record({{cu, {one, 1}}, {cv, {one, 1}}}))) return rc;
  return WAMGPU_OK;
}

template <typename R> std::vector<R> to_r(const float* p, size_t n) {
  std::vector<R> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = R(p[i]);
  return v;
}

template <typename R>
int implsch_host_t(wamgpu_ctx* ctx, Impl<R>& I, float* fl3, const float* u10, const float* udir, float* tauw, float* ustar,
                   float* z0, const float* roairn, const float* wstar, const float* depth, const int* indep) {
  const int n = ctx->nsea;
  const size_t nb = (size_t)n * ctx->cfg.kl * ctx->cfg.ml;
  cudaStream_t s = ctx->stream;
  CK(I.fl3.ensure(nb * sizeof(R)), "alloc");
  for (DevBuf* b : {&I.u10, &I.udir, &I.tauw, &I.ustar, &I.z0, &I.roairn, &I.wstar}) CK(b->ensure((size_t)n * sizeof(R) + 16), "alloc");
  if (depth) { std::vector<R> d = to_r<R>(depth, n); CK(upload(I.d_depth, d, s), "upload depth"); CK(cudaStreamSynchronize(s), "sync"); }
  if (indep) { CK(cudaMemcpyAsync(I.d_indep.p, indep, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s), "upload indep"); }
  struct Up { void* d; const float* h; size_t n; };
  Up ups[] = {{I.fl3.p, fl3, nb}, {I.u10.p, u10, (size_t)n}, {I.udir.p, udir, (size_t)n}, {I.tauw.p, tauw, (size_t)n},
              {I.ustar.p, ustar, (size_t)n}, {I.z0.p, z0, (size_t)n}, {I.roairn.p, roairn, (size_t)n}, {I.wstar.p, wstar, (size_t)n}};
  std::vector<std::vector<R>> keep;
  for (auto& u : ups) {
    if (sizeof(R) == 4) CK(cudaMemcpyAsync(u.d, u.h, u.n * 4, cudaMemcpyHostToDevice, s), "H2D");
    else { keep.push_back(to_r<R>(u.h, u.n)); CK(cudaMemcpyAsync(u.d, keep.back().data(), u.n * sizeof(R), cudaMemcpyHostToDevice, s), "H2D"); }
  }
  int rc = implsch_dev_t<R>(ctx, I, I.fl3.p, n, I.u10.p, I.udir.p, I.tauw.p, I.ustar.p, I.z0.p, I.roairn.p, I.wstar.p, s);
  if (rc) return rc;
  struct Dn { float* h; void* d; size_t n; };
  Dn dns[] = {{fl3, I.fl3.p, nb}, {tauw, I.tauw.p, (size_t)n}, {ustar, I.ustar.p, (size_t)n}, {z0, I.z0.p, (size_t)n}};
  for (auto& d : dns) {
    if (sizeof(R) == 4) CK(cudaMemcpyAsync(d.h, d.d, d.n * 4, cudaMemcpyDeviceToHost, s), "D2H");
    else {
      std::vector<R> tmp(d.n);
      CK(cudaMemcpyAsync(tmp.data(), d.d, d.n * sizeof(R), cudaMemcpyDeviceToHost, s), "D2H");
      CK(cudaStreamSynchronize(s), "sync");
      for (size_t i = 0; i < d.n; ++i) d.h[i] = (float)tmp[i];
    }
  }
  CK(cudaStreamSynchronize(s), "implsch sync");
  return wamgpu_sync(ctx);
}

// Chunks per host<->device copy piece of wamgpu_step_host.  One: pieces of
// 2 and 4 chunks (longer copy rows) made the regional step 1-4 % slower, the
// later first download costing more than the rows gained.
constexpr int kChunksPerCopy = 1;

// Host-buffer form of one WAMODEL pass, with the copies overlapped (see the
// chunk pipeline below).  Results are identical to the unsplit sequence:
// every kernel sees the same inputs and writes the same elements.
template <typename R>
int step_host_t(wamgpu_ctx* ctx, Impl<R>& I, float* fl3, int nprop, const float* u10, const float* udir, float* tauw,
                float* ustar, float* z0, const float* roairn, const float* wstar) {
  static_assert(sizeof(R) == 4 || sizeof(R) == 8, "");
  if (sizeof(R) != 4) return fail(ctx, WAMGPU_E_ARG, "wamgpu_step_host is FP32 only; use wamgpu_step_dev");
  if (!ctx->prepared) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_propagation first");
  if (nprop < 0) return fail(ctx, WAMGPU_E_ARG, "nprop < 0");
  if (ctx->cfg.shallow_run && ctx->cfg.isnonlin != 0 && !I.has_enh)
    return fail(ctx, WAMGPU_E_STATE, "call wamgpu_prepare_source first (ISNONLIN table)");
  const int n = ctx->nsea, KL = ctx->cfg.kl, ML = ctx->cfg.ml;
  const size_t plane = (size_t)n * KL, nb = plane * ML;
  cudaStream_t s = ctx->stream, c = ctx->copy_stream;
  CK(I.fl3.ensure(nb * sizeof(R)), "alloc");
  CK(I.scratch.ensure(nb * sizeof(R)), "alloc scratch");
  for (DevBuf* b : {&I.u10, &I.udir, &I.tauw, &I.ustar, &I.z0, &I.roairn, &I.wstar}) CK(b->ensure((size_t)n * sizeof(R) + 16), "alloc");
  if (!I.status.p) { CK(I.status.ensure(16), "alloc"); CK(cudaMemsetAsync(I.status.p, 0, 16, s), "memset"); }
  if (ctx->cfg.lcflx) CK(I.fluxes.ensure((size_t)7 * n * sizeof(R) + 16), "alloc");
  struct Up { void* d; const float* h; };
  Up ups[] = {{I.u10.p, u10}, {I.udir.p, udir}, {I.tauw.p, tauw}, {I.ustar.p, ustar}, {I.z0.p, z0}, {I.roairn.p, roairn},
              {I.wstar.p, wstar}};
  for (auto& u : ups) CK(cudaMemcpyAsync(u.d, u.h, (size_t)n * 4, cudaMemcpyHostToDevice, s), "H2D");
  R* f3 = I.fl3.template as<R>();
  R* sc = I.scratch.template as<R>();
  const int nsub = nprop * ctx->counter;
  // Chunks of consecutive sea points, each at least as wide as the largest
  // neighbour distance, so that a sub-step of chunk q reads only chunks
  // q-1..q+1.  Chunk q goes up on `c`, is propagated and integrated on `s`
  // and comes down on `d`, so the two copy directions and the kernels overlap.
  // The kernels are issued in the order of the key q + j - 1 (sub-step j of
  // chunk q), ascending j within a key, with IMPLSCH of chunk q last under key
  // q + nsub.  Sub-step j of chunk q then follows sub-step j-1 of chunks
  // q-1..q+1, whose results it reads and whose input buffer it overwrites; it
  // precedes sub-step j+1 of chunk q-1, which overwrites its input; and
  // IMPLSCH of chunk q follows the last sub-step of chunks q-1..q+1.
  const int width = std::max(ctx->halo, 1);
  const int nq = n > 0 ? std::min(64, std::max(1, n / width)) : 1;
  std::vector<int> lo(nq + 1);
  {
    // The first nsub+2 chunks are small (a quarter of the others, and at least
    // one neighbour distance), so that the first IMPLSCH, and with it the
    // first download, starts after a few MB have gone up rather than after
    // nsub+2 full chunks.  The other chunks share the rest evenly.
    const int nsmall = std::min(nq - 1, nsub + 2);
    const int small = std::max(width, n / (4 * nq));
    if (nq > nsmall + 1 && (long long)small * nsmall < n / 2) {
      for (int q = 0; q <= nsmall; ++q) lo[q] = q * small;
      const int rest = n - lo[nsmall], nr = nq - nsmall;
      for (int q = 1; q <= nr; ++q) lo[nsmall + q] = lo[nsmall] + (int)((long long)rest * q / nr);
    } else {
      for (int q = 0; q <= nq; ++q) lo[q] = (int)((long long)n * q / nq);
    }
  }
  // copies move pieces of kChunksPerCopy chunks
  const int cpc = kChunksPerCopy, npc = (nq + cpc - 1) / cpc;
  auto piece_lo = [&](int p) { return lo[std::min(nq, p * cpc)]; };
  const int nev = 2 * npc;
  if ((int)ctx->xfer_ev.size() < nev)
    for (int i = (int)ctx->xfer_ev.size(); i < nev; ++i) {
      cudaEvent_t e;
      CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
      ctx->xfer_ev.push_back(e);
    }
  cudaStream_t d = ctx->down_stream;
  // the spectrum piece by piece (the per-point fields went up on s above)
  for (int p = 0; p < npc; ++p) {
    const int a0 = piece_lo(p);
    const size_t w = (size_t)(piece_lo(p + 1) - a0) * 4;
    if (w) CK(cudaMemcpy2DAsync(f3 + a0, (size_t)n * 4, fl3 + a0, (size_t)n * 4, w, (size_t)KL * ML,
                                cudaMemcpyHostToDevice, c), "H2D");
    CK(cudaEventRecord(ctx->xfer_ev[p], c), "event");
  }
  R* buf[2] = {f3, sc};
  const R* fin = buf[nsub % 2];  // the buffer the last sub-step writes
  auto ready = [&](int q) -> int {  // chunk q and its neighbours are on the device
    CK(cudaStreamWaitEvent(s, ctx->xfer_ev[std::min(q + 1, nq - 1) / cpc], 0), "wait");
    return WAMGPU_OK;
  };
  const int last = (nq - 1) + nsub;
  for (int t = 0; t <= last; ++t) {
    for (int j = 1; j <= nsub; ++j) {
      const int q = t - (j - 1);
      if (q < 0 || q >= nq) continue;
      if (j == 1) { int rc = ready(q); if (rc) return rc; }
      PropArgs<R> A = I.pa;
      A.i0 = lo[q]; A.i1 = lo[q + 1];
      { TimedLaunch tl(ctx, 0, s); CK(launch_propags<R>(A, buf[(j - 1) % 2], n, buf[j % 2], n, s), "propags launch"); }
    }
    const int q = t - nsub;
    if (q < 0 || q >= nq) continue;
    if (nsub == 0) { int rc = ready(q); if (rc) return rc; }
    const int p0 = lo[q], p1 = lo[q + 1];
    if (p1 > p0) {
      ImplArgs<R> a;
      a.nsea = p1 - p0; a.ld = n;
      a.fl3_in = fin + p0; a.fl3 = f3 + p0;
      a.u10 = I.u10.template as<R>() + p0; a.udir = I.udir.template as<R>() + p0;
      a.roairn = I.roairn.template as<R>() + p0; a.wstar = I.wstar.template as<R>() + p0;
      a.depth = I.d_depth.template as<R>() + p0; a.indep = I.d_indep.template as<int>() + p0;
      a.tauw = I.tauw.template as<R>() + p0; a.ustar = I.ustar.template as<R>() + p0; a.z0 = I.z0.template as<R>() + p0;
      a.fluxes = ctx->cfg.lcflx ? I.fluxes.template as<R>() + p0 : nullptr;
      a.flx_ld = n;
      a.status = I.status.template as<int>();
      a.enh = I.has_enh ? I.enh.template as<R>() + p0 : nullptr; a.enh_ld = n;
      a.wncg = ctx->wncg_valid ? I.wncg.template as<R>() + (size_t)p0 * 2 * ctx->cfg.ml : nullptr;
      { TimedLaunch tl(ctx, 1, s); CK(launch_implsch<R>(I.dt, a, ctx->P, s), "implsch launch"); }
    }
    if (q % cpc == cpc - 1 || q == nq - 1) {  // the last chunk of a piece: the piece goes down
      const int pc = q / cpc, a0 = piece_lo(pc);
      CK(cudaEventRecord(ctx->xfer_ev[npc + pc], s), "event");
      CK(cudaStreamWaitEvent(d, ctx->xfer_ev[npc + pc], 0), "wait");
      const size_t w = (size_t)(piece_lo(pc + 1) - a0) * 4;
      if (w) CK(cudaMemcpy2DAsync(fl3 + a0, (size_t)n * 4, f3 + a0, (size_t)n * 4, w, (size_t)KL * ML,
                                  cudaMemcpyDeviceToHost, d), "D2H");
    }
  }
  // TAUW, USTAR, Z0 after the last piece (d follows the last IMPLSCH)
  CK(cudaMemcpyAsync(tauw, I.tauw.template as<R>(), (size_t)n * 4, cudaMemcpyDeviceToHost, d), "D2H");
  CK(cudaMemcpyAsync(ustar, I.ustar.template as<R>(), (size_t)n * 4, cudaMemcpyDeviceToHost, d), "D2H");
  CK(cudaMemcpyAsync(z0, I.z0.template as<R>(), (size_t)n * 4, cudaMemcpyDeviceToHost, d), "D2H");
  CK(cudaStreamSynchronize(d), "step copies");
  CK(cudaStreamSynchronize(c), "step copies");
  CK(cudaStreamSynchronize(s), "step sync");
  return wamgpu_sync(ctx);
}

template <typename R> int propags_host_t(wamgpu_ctx* ctx, Impl<R>& I, float* f3) {
  const size_t nb = (size_t)ctx->nsea * ctx->cfg.kl * ctx->cfg.ml;
  cudaStream_t s = ctx->stream;
  CK(I.fl3.ensure(nb * sizeof(R)), "alloc");
  std::vector<R> tmp;
  if (sizeof(R) == 4) CK(cudaMemcpyAsync(I.fl3.p, f3, nb * 4, cudaMemcpyHostToDevice, s), "H2D");
  else { tmp = to_r<R>(f3, nb); CK(cudaMemcpyAsync(I.fl3.p, tmp.data(), nb * sizeof(R), cudaMemcpyHostToDevice, s), "H2D"); }
  int rc = propags_dev_t<R>(ctx, I, I.fl3.p, ctx->nsea, nullptr, s);
  if (rc) return rc;
  if (sizeof(R) == 4) CK(cudaMemcpyAsync(f3, I.fl3.p, nb * 4, cudaMemcpyDeviceToHost, s), "D2H");
  else {
    CK(cudaMemcpyAsync(tmp.data(), I.fl3.p, nb * sizeof(R), cudaMemcpyDeviceToHost, s), "D2H");
    CK(cudaStreamSynchronize(s), "sync");
    for (size_t i = 0; i < nb; ++i) f3[i] = (float)tmp[i];
  }
  CK(cudaStreamSynchronize(s), "propags sync");
  return WAMGPU_OK;
}

template <typename R> int get_table_t(const wamgpu_ctx* ctx, const Impl<R>& I, const std::string& n, float* fo, int* io) {
  const TableSet<R>& t = I.tab;
  const std::vector<R>* f = nullptr; const std::vector<int>* iv = nullptr;
  std::vector<R> tmp; std::vector<int> itmp;
  if (n == "FR") f = &t.FR; else if (n == "DF") f = &t.DF; else if (n == "DFIM") f = &t.DFIM; else if (n == "GOM") f = &t.GOM;
  else if (n == "C") f = &t.C; else if (n == "TH") f = &t.TH; else if (n == "COSTH") f = &t.COSTH; else if (n == "SINTH") f = &t.SINTH;
  else if (n == "DFIMOFR") f = &t.DFIMOFR; else if (n == "FR5") f = &t.FR5; else if (n == "FRM5") f = &t.FRM5;
  else if (n == "RHOWG_DFIM") f = &t.RHOWG_DFIM; else if (n == "TFAK") f = &t.TFAK; else if (n == "TCGOND") f = &t.TCGOND;
  else if (n == "TSIHKD") f = &t.TSIHKD; else if (n == "FLMINFR") f = &t.FLMINFR; else if (n == "AF11") f = &t.AF11;
  else if (n == "FKLAP") f = &t.FKLAP; else if (n == "FKLAP1") f = &t.FKLAP1; else if (n == "FKLAM") f = &t.FKLAM;
  else if (n == "FKLAM1") f = &t.FKLAM1; else if (n == "FRH") f = &t.FRH; else if (n == "RNLCOEF") f = &t.RNLCOEF;
  else if (n == "SWELLFT") f = &t.SWELLFT; else if (n == "SATWEIGHTS") f = &t.SATWEIGHTS; else if (n == "WTAUHF") f = &t.WTAUHF;
  else if (n == "SCALARS") {
    tmp = {t.DELTH, t.DELTR, t.INV_LOG_CO, t.MO_TAIL, t.MM1_TAIL, t.MP1_TAIL, R(0), R(0), t.DELU, t.ACL1, t.ACL2, t.CL11,
           t.CL21, t.DAL1, t.DAL2, t.X0TAUHF};
    f = &tmp;
  } else if (n == "IKP") iv = &t.IKP; else if (n == "IKP1") iv = &t.IKP1; else if (n == "IKM") iv = &t.IKM;
  else if (n == "IKM1") iv = &t.IKM1; else if (n == "K1W") iv = &t.K1W; else if (n == "K2W") iv = &t.K2W;
  else if (n == "K11W") iv = &t.K11W; else if (n == "K21W") iv = &t.K21W; else if (n == "INLCOEF") iv = &t.INLCOEF;
  else if (n == "INDICESSAT") iv = &t.INDICESSAT;
  else if (n == "DIA_SCALARS") { itmp = {t.MFRSTLW, t.MLSTHG, t.KFRH, 0, 0, t.NSDSNTH}; iv = &itmp; }
  else if (n == "INDEP") iv = &ctx->indep;
  if (f) { if (fo) for (size_t i = 0; i < f->size(); ++i) fo[i] = (float)(*f)[i]; return (int)f->size(); }
  if (iv) { if (io) std::memcpy(io, iv->data(), iv->size() * sizeof(int)); return (int)iv->size(); }
  return WAMGPU_E_ARG;
}

// ---- batched ensembles -------------------------------------------------------
// Many member contexts (uneven NSEA, mixed KL/ML/IPHYS, one precision, one
// device) advance together: each PROPAGS sub-step is one launch per
// coefficient family over all members that still have that sub-step, and
// IMPLSCH is one launch over all members.  The launch lists live on the
// device, so a pass is a fixed sequence of launches that can be captured
// once as a CUDA graph and replayed.
struct BatchState {
  void* fl3 = nullptr; void* scratch = nullptr; int ld = 0;
  const void *u10 = nullptr, *udir = nullptr, *roairn = nullptr, *wstar = nullptr;
  void *tauw = nullptr, *ustar = nullptr, *z0 = nullptr;
};
struct BatchList { int family = 0; int nmem = 0, nblocks = 0, P = 0; size_t smem = 0; DevBuf mem, first; };

}  // namespace

struct wamgpu_batch {
  std::string err;
  std::vector<wamgpu_ctx*> members;
  int precision = 4, device = 0;
  std::vector<BatchState> st;
  std::vector<int> Pc;  // IMPLSCH sea points per CTA of each source-table class (empty: the contexts' own choice)
  int bs = 128;         // PROPAGS points per CTA
  bool built = false;
  std::vector<std::vector<BatchList>> sub;  // [sub-step][family group]
  std::vector<BatchList> imp;               // IMPLSCH, one list per shared-memory class
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t stream = nullptr;
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr; graph = nullptr;
  }
};

namespace {

int bfail(wamgpu_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}
#define BCK(call, where)                                                                    \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) return bfail(b, WAMGPU_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T> cudaError_t upload_vec(DevBuf& d, const std::vector<T>& h, cudaStream_t s) {
  cudaError_t e = d.ensure(h.size() * sizeof(T) + 16);
  if (e != cudaSuccess || h.empty()) return e;
  return cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

template <typename R> Impl<R>& impl_of(wamgpu_ctx* c) { return *static_cast<Impl<R>*>(c->impl.get()); }

// sub-steps of a member in one pass: IDELT/IDELPRO propagation calls of COUNTER sub-steps each
int member_nsub(const wamgpu_ctx* c) { return (c->cfg.idelt / c->cfg.idelpro) * c->counter; }

constexpr size_t kMaxSmemPerCta = 232448;  // 227 KB opt-in limit of sm_100

// The configuration fields that determine a context's source tables
// (DevTables): members that agree on them can share one batched IMPLSCH
// launch with one member's tables as the kernel parameter.
std::vector<double> source_key(const Config& c) {
  return {double(c.kl), double(c.ml), c.fr1, double(c.iref), double(c.iphys), double(c.shallow_run),
          double(c.isnonlin), double(c.lcflx), double(c.idelt), c.betamax, c.zalp, c.alpha, c.tauwshelter, c.cdfac,
          double(c.ndepth), c.deptha, c.depthd, double(c.precision)};
}

// IMPLSCH member lists, one per source-table class, largest members first
// (their CTAs start first).  For tuning (out != null) each member reads its
// current spectrum and writes `out`, TAUW/USTAR/Z0 go to `tmp3` and the
// status flag to `tmp_status`: the members' state is left untouched.
template <typename R>
int batch_impl_lists(wamgpu_batch* b, const std::vector<int>& Pin, std::vector<BatchList>& Ls, const std::vector<R*>* out,
                     const std::vector<R*>* tmp3, int* tmp_status, cudaStream_t s) {
  const int n = (int)b->members.size();
  std::vector<std::vector<double>> keys;
  std::vector<int> cls(n);
  for (int g = 0; g < n; ++g) {
    std::vector<double> k = source_key(b->members[g]->cfg);
    auto it = std::find(keys.begin(), keys.end(), k);
    cls[g] = (int)(it - keys.begin());
    if (it == keys.end()) keys.push_back(k);
  }
  Ls.clear();
  Ls.resize(keys.size());
  for (size_t ci = 0; ci < keys.size(); ++ci) {
    std::vector<int> order;
    for (int g = 0; g < n; ++g) if (cls[g] == (int)ci) order.push_back(g);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->members[x]->nsea > b->members[y]->nsea; });
    // sea points per CTA: the tuned value of this class, else the contexts' own occupancy choice
    const int P = (ci < Pin.size() && Pin[ci] > 0) ? Pin[ci] : b->members[order[0]]->P;
    if (implsch_smem_bytes(impl_of<R>(b->members[order[0]]).dt, P) + sizeof(ImplArgs<R>) + 64 > kMaxSmemPerCta)
      return bfail(b, WAMGPU_E_ARG, "points per CTA too large for a member");
    std::vector<ImplArgs<R>> mem(order.size());
    std::vector<int> first(order.size() + 1, 0);
    for (size_t q = 0; q < order.size(); ++q) {
      const int g = order[q];
      wamgpu_ctx* c = b->members[g];
      Impl<R>& I = impl_of<R>(c);
      const BatchState& x = b->st[g];
      if (!I.status.p) { BCK(I.status.ensure(16), "alloc"); BCK(cudaMemsetAsync(I.status.p, 0, 16, s), "memset"); }
      if (c->cfg.lcflx) BCK(I.fluxes.ensure((size_t)7 * c->nsea * sizeof(R) + 16), "alloc");
      ImplArgs<R>& a = mem[q];
      a.nsea = c->nsea; a.ld = x.ld;
      R* fin = (member_nsub(c) % 2 == 0) ? (R*)x.fl3 : (R*)x.scratch;  // buffer the last sub-step wrote
      a.fl3_in = out ? (const R*)x.fl3 : fin;
      a.fl3 = out ? (*out)[g] : (R*)x.fl3;
      a.u10 = (const R*)x.u10; a.udir = (const R*)x.udir; a.roairn = (const R*)x.roairn; a.wstar = (const R*)x.wstar;
      a.depth = I.d_depth.template as<R>(); a.indep = I.d_indep.template as<int>();
      if (tmp3) { a.tauw = (*tmp3)[3 * g]; a.ustar = (*tmp3)[3 * g + 1]; a.z0 = (*tmp3)[3 * g + 2]; }
      else { a.tauw = (R*)x.tauw; a.ustar = (R*)x.ustar; a.z0 = (R*)x.z0; }
      a.fluxes = (c->cfg.lcflx && !tmp3) ? I.fluxes.template as<R>() : nullptr;
      a.flx_ld = c->nsea;
      a.enh = I.has_enh ? I.enh.template as<R>() : nullptr; a.enh_ld = c->nsea;
      a.wncg = c->wncg_valid ? I.wncg.template as<R>() : nullptr;
      a.status = tmp_status ? tmp_status : I.status.template as<int>();
      first[q + 1] = first[q] + (c->nsea + P - 1) / P;
    }
    BatchList& L = Ls[ci];
    L.family = order[0];  // whose source tables the launch passes
    L.P = P;
    L.smem = implsch_smem_bytes(impl_of<R>(b->members[order[0]]).dt, P);
    BCK(implsch_set_max_smem<R>(P, L.smem), "smem attribute");
    BCK(upload_vec(L.mem, mem, s), "upload batch");
    BCK(upload_vec(L.first, first, s), "upload batch");
    L.nmem = (int)order.size(); L.nblocks = first.back();
  }
  return WAMGPU_OK;
}

template <typename R> int launch_impl_lists(wamgpu_batch* b, const std::vector<BatchList>& Ls, cudaStream_t s) {
  for (const BatchList& L : Ls)
    BCK(launch_implsch_batch<R>(impl_of<R>(b->members[L.family]).dt, L.mem.template as<ImplArgs<R>>(),
                                L.first.template as<int>(), L.nmem, L.nblocks, L.P, L.smem, s), "batched IMPLSCH");
  return WAMGPU_OK;
}

template <typename R> int batch_build(wamgpu_batch* b, cudaStream_t s) {
  const int n = (int)b->members.size();
  for (int g = 0; g < n; ++g)
    if (!b->st[g].fl3) return bfail(b, WAMGPU_E_STATE, "member " + std::to_string(g) + " has no state (wamgpu_batch_set_member)");
  int maxsub = 0;
  for (auto* c : b->members) maxsub = std::max(maxsub, member_nsub(c));
  b->sub.clear();
  b->sub.resize(maxsub);
  auto key_of = [](const PropArgs<R>& A) { return A.variant * 4 + (A.reduced ? 2 : 0) + (A.refr_d ? 1 : 0); };
  for (int it = 0; it < maxsub; ++it) {
    std::vector<int> fam;  // coefficient families in order of first appearance
    for (int g = 0; g < n; ++g) {
      wamgpu_ctx* c = b->members[g];
      if (member_nsub(c) <= it || c->nsea == 0) continue;
      const int key = key_of(impl_of<R>(c).pa);
      if (std::find(fam.begin(), fam.end(), key) == fam.end()) fam.push_back(key);
    }
    b->sub[it].resize(fam.size());
    for (size_t f = 0; f < fam.size(); ++f) {
      std::vector<PropMember<R>> mem;
      std::vector<int> first(1, 0);
      int rep = -1;
      for (int g = 0; g < n; ++g) {
        wamgpu_ctx* c = b->members[g];
        if (member_nsub(c) <= it || c->nsea == 0) continue;
        const PropArgs<R>& A = impl_of<R>(c).pa;
        if (key_of(A) != fam[f]) continue;
        if (rep < 0) rep = g;
        PropMember<R> M;
        M.A = A;
        R* f3 = (R*)b->st[g].fl3; R* sc = (R*)b->st[g].scratch;
        M.src = (it % 2 == 0) ? f3 : sc;
        M.dst = (it % 2 == 0) ? sc : f3;
        M.ld = b->st[g].ld;
        M.nbi = (A.i1 - A.i0 + b->bs - 1) / b->bs;
        mem.push_back(M);
        first.push_back(first.back() + c->cfg.ml * M.nbi);
      }
      BatchList& L = b->sub[it][f];
      L.family = rep;
      L.nmem = (int)mem.size(); L.nblocks = first.back();
      BCK(upload_vec(L.mem, mem, s), "upload batch");
      BCK(upload_vec(L.first, first, s), "upload batch");
    }
  }
  int rc = batch_impl_lists<R>(b, b->Pc, b->imp, nullptr, nullptr, nullptr, s);
  if (rc) return rc;

  BCK(cudaStreamSynchronize(s), "batch upload");
  b->built = true;
  return WAMGPU_OK;
}

template <typename R> int batch_launch(wamgpu_batch* b, cudaStream_t s) {
  for (auto& step : b->sub)
    for (auto& L : step) {
      const PropArgs<R>& fam = impl_of<R>(b->members[L.family]).pa;
      BCK(launch_propags_batch<R>(fam, L.mem.template as<PropMember<R>>(), L.first.template as<int>(), L.nmem, L.nblocks,
                                  b->bs, s), "batched PROPAGS");
    }
  return launch_impl_lists<R>(b, b->imp, s);
}

// Autotuner: times the first batched PROPAGS sub-step with 128- and 256-point
// CTAs (it reads FL3 and writes scratch only) and the batched IMPLSCH for
// every compiled CTA shape out of place (spectra into scratch, TAUW/USTAR/Z0
// and the status flag into temporaries), and keeps the fastest of each.
template <typename R> int batch_tune(wamgpu_batch* b, cudaStream_t s, int* P_out, int* bs_out) {
  const int n = (int)b->members.size();
  b->drop_graph();
  b->built = false;
  int rc = batch_build<R>(b, s);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0), "event");
  BCK(cudaEventCreate(&e1), "event");
  auto timed = [&](auto&& launch, float& best) -> int {
    best = 1e30f;
    for (int r = 0; r < 4; ++r) {
      BCK(cudaEventRecord(e0, s), "event");
      int rc2 = launch();
      if (rc2) return rc2;
      BCK(cudaEventRecord(e1, s), "event");
      BCK(cudaEventSynchronize(e1), "event");
      float ms = 0;
      BCK(cudaEventElapsedTime(&ms, e0, e1), "event");
      if (r > 0) best = std::min(best, ms);
    }
    return WAMGPU_OK;
  };
  int best_bs = b->bs;
  float best_t = 1e30f;
  for (int cand : {128, 256}) {
    b->bs = cand; b->built = false;
    if ((rc = batch_build<R>(b, s))) break;
    if (b->sub.empty()) { best_bs = cand; break; }
    float t = 0;
    rc = timed([&]() -> int {
      for (auto& L : b->sub[0]) {
        const PropArgs<R>& fam = impl_of<R>(b->members[L.family]).pa;
        BCK(launch_propags_batch<R>(fam, L.mem.template as<PropMember<R>>(), L.first.template as<int>(), L.nmem, L.nblocks,
                                    b->bs, s), "batched PROPAGS");
      }
      return WAMGPU_OK;
    }, t);
    if (rc) break;
    if (t < best_t) { best_t = t; best_bs = cand; }
  }
  b->bs = best_bs;
  DevBuf tmp, tstatus;
  size_t tot = 0;
  for (auto* c : b->members) tot += (size_t)c->nsea + 4;
  if (!rc && tmp.ensure(3 * tot * sizeof(R) + 64) != cudaSuccess) rc = bfail(b, WAMGPU_E_NOMEM, "tuning buffers");
  if (!rc && tstatus.ensure(16) != cudaSuccess) rc = bfail(b, WAMGPU_E_NOMEM, "tuning buffers");
  std::vector<R*> out(n), t3(3 * n);
  if (!rc) {
    size_t off = 0;
    for (int g = 0; g < n && !rc; ++g) {
      const size_t ng = (size_t)b->members[g]->nsea;
      out[g] = (R*)b->st[g].scratch;
      for (int q = 0; q < 3; ++q) {
        t3[3 * g + q] = tmp.template as<R>() + off;
        const void* srcp = q == 0 ? b->st[g].tauw : (q == 1 ? b->st[g].ustar : b->st[g].z0);
        if (ng && cudaMemcpyAsync(t3[3 * g + q], srcp, ng * sizeof(R), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
          rc = bfail(b, WAMGPU_E_CUDA, "tuning copy");
          break;
        }
        off += ng + 4;
      }
    }
  }
  // IMPLSCH: each source-table class keeps its fastest CTA shape
  const size_t ncls = b->imp.size();
  std::vector<int> bestP(ncls, 0);
  std::vector<float> bestT(ncls, 1e30f);
  const std::vector<int> cands = sizeof(R) == 4 ? std::vector<int>{4, 6, 8} : std::vector<int>{2, 4};
  for (int P : cands) {
    if (rc) break;
    std::vector<int> Pin(ncls, P);
    for (size_t ci = 0; ci < ncls; ++ci)  // classes this shape does not fit keep their default
      if (implsch_smem_bytes(impl_of<R>(b->members[b->imp[ci].family]).dt, P) + sizeof(ImplArgs<R>) + 64 > kMaxSmemPerCta)
        Pin[ci] = 0;
    std::vector<BatchList> Ls;
    if ((rc = batch_impl_lists<R>(b, Pin, Ls, &out, &t3, tstatus.template as<int>(), s))) break;
    for (size_t ci = 0; ci < ncls && !rc; ++ci) {
      if (Pin[ci] == 0) continue;
      float t = 0;
      std::vector<BatchList> one(1);
      one[0].family = Ls[ci].family; one[0].nmem = Ls[ci].nmem; one[0].nblocks = Ls[ci].nblocks; one[0].P = Ls[ci].P;
      one[0].smem = Ls[ci].smem;
      one[0].mem = std::move(Ls[ci].mem); one[0].first = std::move(Ls[ci].first);
      rc = timed([&]() -> int { return launch_impl_lists<R>(b, one, s); }, t);
      if (!rc && t < bestT[ci]) { bestT[ci] = t; bestP[ci] = P; }
    }
    BCK(cudaStreamSynchronize(s), "tune");
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  b->Pc = bestP;
  b->built = false;
  if ((rc = batch_build<R>(b, s))) return rc;
  if (P_out) {  // the shape of the class with the most sea points
    size_t best = 0; int pc = b->imp.empty() ? 0 : b->imp[0].P;
    for (size_t ci = 0; ci < b->imp.size(); ++ci) {
      size_t pts = 0;
      for (size_t g = 0; g < b->members.size(); ++g)
        if (source_key(b->members[g]->cfg) == source_key(b->members[b->imp[ci].family]->cfg)) pts += b->members[g]->nsea;
      if (pts > best) { best = pts; pc = b->imp[ci].P; }
    }
    *P_out = pc;
  }
  if (bs_out) *bs_out = b->bs;
  return WAMGPU_OK;
}

#define DISPATCH_CTX(ctx, FN, ...)                                                              \
  ((ctx)->cfg.precision == 8 ? FN<double>((ctx), *static_cast<Impl<double>*>((ctx)->impl.get()), ##__VA_ARGS__) \
                             : FN<float>((ctx), *static_cast<Impl<float>*>((ctx)->impl.get()), ##__VA_ARGS__))

}  // namespace

extern "C" {

int wamgpu_config_size(void) { return (int)sizeof(wamgpu_config); }

int wamgpu_create(const wamgpu_config* cfg, wamgpu_ctx** out) {
  if (!cfg || !out) return WAMGPU_E_ARG;
  *out = nullptr;
  auto* ctx = new wamgpu_ctx();
  ctx->cfg = *cfg;
  const Config& c = ctx->cfg;
  auto bail = [&](int rc) { if (rc) { /* keep ctx for wamgpu_last_error */ *out = ctx; } return rc; };
  if (c.kl < 4 || c.kl > MAX_KL || c.ml < 4 || c.ml > MAX_ML) return bail(fail(ctx, WAMGPU_E_ARG, "KL/ML outside supported range"));
  if (c.iphys != 1 && c.iphys != 2) return bail(fail(ctx, WAMGPU_E_ARG, "only IPHYS=1 (ST4) and IPHYS=2 (ST6) are implemented"));
  if (c.precision != 4 && c.precision != 8) return bail(fail(ctx, WAMGPU_E_ARG, "precision must be 4 or 8"));
  if (c.idelt <= 0 || c.idelpro <= 0) return bail(fail(ctx, WAMGPU_E_ARG, "time steps must be positive"));
  if (c.refraction_c_run && !c.refraction_d_run && c.shallow_run)
    return bail(fail(ctx, WAMGPU_E_ARG, "current refraction requires depth refraction (SET_MODEL_OPTION)"));
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return bail(fail(ctx, WAMGPU_E_CUDA, "no CUDA device: libwamgpu has no CPU path"));
  if (c.device < 0 || c.device >= ndev) return bail(fail(ctx, WAMGPU_E_ARG, "device ordinal out of range"));
  if ((e = cudaSetDevice(c.device)) != cudaSuccess) return bail(cuda_fail(ctx, e, "cudaSetDevice"));
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(cuda_fail(ctx, e, "stream"));
  if ((e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(cuda_fail(ctx, e, "stream"));
  if ((e = cudaStreamCreateWithFlags(&ctx->down_stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(cuda_fail(ctx, e, "stream"));
  cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, c.device);
  int rc;
  if (c.precision == 8) { auto* I = new Impl<double>(); ctx->impl.reset(I); rc = build_tables<double>(ctx, *I); }
  else { auto* I = new Impl<float>(); ctx->impl.reset(I); rc = build_tables<float>(ctx, *I); }
  if (rc) return bail(rc);
  *out = ctx;
  return WAMGPU_OK;
}

int wamgpu_destroy(wamgpu_ctx* ctx) {
  if (!ctx) return WAMGPU_OK;
  if (ctx->stream) { cudaSetDevice(ctx->cfg.device); cudaStreamSynchronize(ctx->stream); }
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  if (ctx->down_stream) cudaStreamSynchronize(ctx->down_stream);
  ctx->impl.reset();
  for (int c = 0; c < 2; ++c) for (auto& e : ctx->ev[c]) ctx->ev_pool.push_back(e);
  for (auto& e : ctx->ev_pool) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  for (auto e : ctx->xfer_ev) cudaEventDestroy(e);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->down_stream) cudaStreamDestroy(ctx->down_stream);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return WAMGPU_OK;
}

const char* wamgpu_last_error(const wamgpu_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int wamgpu_get_table(const wamgpu_ctx* ctx, const char* name, float* fout, int* iout) {
  if (!ctx || !name || !ctx->impl) return WAMGPU_E_ARG;
  std::string n(name);
  if (ctx->cfg.precision == 8) return get_table_t<double>(ctx, *static_cast<Impl<double>*>(ctx->impl.get()), n, fout, iout);
  return get_table_t<float>(ctx, *static_cast<Impl<float>*>(ctx->impl.get()), n, fout, iout);
}

int wamgpu_host_table(const wamgpu_config* cfg, const char* name, float* fout, int* iout) {
  if (!cfg || !name) return WAMGPU_E_ARG;
  if (cfg->kl < 4 || cfg->kl > MAX_KL || cfg->ml < 4 || cfg->ml > MAX_ML) return WAMGPU_E_ARG;
  wamgpu_ctx tmp;
  tmp.cfg = *cfg;
  std::string n(name);
  if (cfg->precision == 8) {
    Impl<double> I; I.tab.build(*cfg);
    return get_table_t<double>(&tmp, I, n, fout, iout);
  }
  Impl<float> I; I.tab.build(*cfg);
  return get_table_t<float>(&tmp, I, n, fout, iout);
}

int wamgpu_set_grid(wamgpu_ctx* ctx, int nsea, const int* klat, const int* klon, const float* wlat, const int* kfromij,
                    int ny, const float* sinph, const float* cosph, const float* dellam) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (nsea < 0 || ny <= 0 || (nsea > 0 && (!klat || !klon || !wlat || !kfromij)) || !sinph || !cosph || !dellam)
    return fail(ctx, WAMGPU_E_ARG, "invalid grid arguments");
  for (int i = 0; i < 4 * nsea; ++i) if (klat[i] < 0 || klat[i] > nsea) return fail(ctx, WAMGPU_E_ARG, "KLAT index out of range");
  for (int i = 0; i < 2 * nsea; ++i) if (klon[i] < 0 || klon[i] > nsea) return fail(ctx, WAMGPU_E_ARG, "KLON index out of range");
  for (int i = 0; i < nsea; ++i) if (kfromij[i] < 1 || kfromij[i] > ny) return fail(ctx, WAMGPU_E_ARG, "KFROMIJ out of range");
  ctx->nsea = nsea; ctx->ny = ny; ctx->n_ext = nsea;
  ctx->halo = 0;
  for (int q = 0; q < 4; ++q)
    for (int i = 0; i < nsea; ++i) { const int p = klat[i + (size_t)nsea * q]; if (p > 0) ctx->halo = std::max(ctx->halo, std::abs(p - 1 - i)); }
  for (int q = 0; q < 2; ++q)
    for (int i = 0; i < nsea; ++i) { const int p = klon[i + (size_t)nsea * q]; if (p > 0) ctx->halo = std::max(ctx->halo, std::abs(p - 1 - i)); }
  ctx->klat.assign(klat, klat + 4 * (size_t)nsea); ctx->klon.assign(klon, klon + 2 * (size_t)nsea);
  ctx->wlat.assign(wlat, wlat + 2 * (size_t)nsea); ctx->kfromij.assign(kfromij, kfromij + nsea);
  ctx->sinph.assign(sinph, sinph + ny); ctx->cosph.assign(cosph, cosph + ny); ctx->dellam.assign(dellam, dellam + ny);
  ctx->depth.assign(nsea, 999.0f); ctx->u.assign(nsea, 0.f); ctx->v.assign(nsea, 0.f);
  ctx->have_grid = true; ctx->prepared = false; ctx->wncg_valid = false;
  ctx->own0 = 0; ctx->own1 = -1;
  cudaSetDevice(ctx->cfg.device);
  return DISPATCH_CTX(ctx, set_grid_t);
}

int wamgpu_set_depth(wamgpu_ctx* ctx, const float* depth) {
  if (!ctx || !ctx->have_grid || !depth) return ctx ? fail(ctx, WAMGPU_E_STATE, "set_grid first") : WAMGPU_E_ARG;
  for (int i = 0; i < ctx->nsea; ++i)
    if (!(depth[i] > 0.f) || !std::isfinite(depth[i])) return fail(ctx, WAMGPU_E_ARG, "depth must be positive and finite");
  ctx->depth.assign(depth, depth + ctx->nsea);
  ctx->prepared = false;
  ctx->wncg_valid = false;
  return WAMGPU_OK;
}

int wamgpu_set_current(wamgpu_ctx* ctx, const float* u, const float* v) {
  if (!ctx || !ctx->have_grid) return ctx ? fail(ctx, WAMGPU_E_STATE, "set_grid first") : WAMGPU_E_ARG;
  if (u) ctx->u.assign(u, u + ctx->nsea); else ctx->u.assign(ctx->nsea, 0.f);
  if (v) ctx->v.assign(v, v + ctx->nsea); else ctx->v.assign(ctx->nsea, 0.f);
  ctx->prepared = false;
  return WAMGPU_OK;
}

int wamgpu_prepare_propagation(wamgpu_ctx* ctx, float* total_cfl, int* counter) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (!ctx->have_grid) return fail(ctx, WAMGPU_E_STATE, "set_grid first");
  cudaSetDevice(ctx->cfg.device);
  return DISPATCH_CTX(ctx, prepare_prop, total_cfl, counter);
}

int wamgpu_prepare_source(wamgpu_ctx* ctx) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (!ctx->have_grid) return fail(ctx, WAMGPU_E_STATE, "set_grid first");
  cudaSetDevice(ctx->cfg.device);
  return DISPATCH_CTX(ctx, prepare_source_t);
}

int wamgpu_get_indep(const wamgpu_ctx* ctx, int* indep) {
  if (!ctx || !indep || !ctx->prepared) return WAMGPU_E_STATE;
  std::memcpy(indep, ctx->indep.data(), ctx->indep.size() * sizeof(int));
  return WAMGPU_OK;
}

int wamgpu_implsch_host(wamgpu_ctx* ctx, float* fl3, const float* u10, const float* udir, float* tauw, float* ustar,
                        float* z0, const float* roairn, const float* wstar, const float* depth, const int* indep) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (!fl3 || !u10 || !udir || !tauw || !ustar || !z0 || !roairn || !wstar) return fail(ctx, WAMGPU_E_ARG, "null argument");
  cudaSetDevice(ctx->cfg.device);
  return DISPATCH_CTX(ctx, implsch_host_t, fl3, u10, udir, tauw, ustar, z0, roairn, wstar, depth, indep);
}

int wamgpu_propags_host(wamgpu_ctx* ctx, float* f3) {
  if (!ctx || !ctx->impl || !f3) return WAMGPU_E_ARG;
  cudaSetDevice(ctx->cfg.device);
  return DISPATCH_CTX(ctx, propags_host_t, f3);
}

int wamgpu_implsch_dev(wamgpu_ctx* ctx, void* fl3, int ld, const void* u10, const void* udir, void* tauw, void* ustar,
                       void* z0, const void* roairn, const void* wstar, void* stream) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (!fl3 || !u10 || !udir || !tauw || !ustar || !z0 || !roairn || !wstar) return fail(ctx, WAMGPU_E_ARG, "null argument");
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, implsch_dev_t, fl3, ld, u10, udir, tauw, ustar, z0, roairn, wstar, s);
}

int wamgpu_propags_dev(wamgpu_ctx* ctx, void* f3, int ld, void* scratch, void* stream) {
  if (!ctx || !ctx->impl || !f3) return WAMGPU_E_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, propags_dev_t, f3, ld, scratch, s);
}

int wamgpu_propags_dev_static(wamgpu_ctx* ctx, void* f3, int ld, void* stream) {
  if (!ctx || !ctx->impl || !f3) return WAMGPU_E_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, propags_dev_static_t, f3, ld, s);
}

int wamgpu_step_dev(wamgpu_ctx* ctx, void* fl3, int ld, void* scratch, int nprop, const void* u10, const void* udir,
                    void* tauw, void* ustar, void* z0, const void* roairn, const void* wstar, void* stream) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (!fl3 || !u10 || !udir || !tauw || !ustar || !z0 || !roairn || !wstar) return fail(ctx, WAMGPU_E_ARG, "null argument");
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, step_dev_t, fl3, ld, scratch, nprop, u10, udir, tauw, ustar, z0, roairn, wstar, s);
}

int wamgpu_step_host(wamgpu_ctx* ctx, float* fl3, int nprop, const float* u10, const float* udir, float* tauw,
                     float* ustar, float* z0, const float* roairn, const float* wstar) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (!fl3 || !u10 || !udir || !tauw || !ustar || !z0 || !roairn || !wstar) return fail(ctx, WAMGPU_E_ARG, "null argument");
  cudaSetDevice(ctx->cfg.device);
  return DISPATCH_CTX(ctx, step_host_t, fl3, nprop, u10, udir, tauw, ustar, z0, roairn, wstar);
}

int wamgpu_get_fluxes(wamgpu_ctx* ctx, float* out7) {
  if (!ctx || !ctx->impl || !out7) return WAMGPU_E_ARG;
  if (!ctx->cfg.lcflx) return fail(ctx, WAMGPU_E_STATE, "LCFLX is off");
  size_t n = (size_t)7 * ctx->nsea;
  cudaSetDevice(ctx->cfg.device);
  if (ctx->cfg.precision == 8) {
    auto* I = static_cast<Impl<double>*>(ctx->impl.get());
    std::vector<double> t(n);
    CK(cudaMemcpyAsync(t.data(), I->fluxes.p, n * 8, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    for (size_t i = 0; i < n; ++i) out7[i] = (float)t[i];
  } else {
    auto* I = static_cast<Impl<float>*>(ctx->impl.get());
    CK(cudaMemcpyAsync(out7, I->fluxes.p, n * 4, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
  }
  return WAMGPU_OK;
}

int wamgpu_set_timing(wamgpu_ctx* ctx, int enable) {
  if (!ctx) return WAMGPU_E_ARG;
  ctx->timing = enable != 0;
  return WAMGPU_OK;
}

int wamgpu_get_timing(wamgpu_ctx* ctx, float* ms, int* count) {
  if (!ctx || !ms || !count) return WAMGPU_E_ARG;
  cudaSetDevice(ctx->cfg.device);
  for (int c = 0; c < 2; ++c) {
    ms[c] = 0.f; count[c] = (int)ctx->ev[c].size();
    for (auto& e : ctx->ev[c]) {
      float t = 0.f;
      CK(cudaEventSynchronize(e.second), "timing");
      CK(cudaEventElapsedTime(&t, e.first, e.second), "timing");
      ms[c] += t;
      ctx->ev_pool.push_back(e);
    }
    ctx->ev[c].clear();
  }
  return WAMGPU_OK;
}

int wamgpu_output_parameters_dev(wamgpu_ctx* ctx, const void* fl3, int ld, const void* u10, const void* udir,
                                 const void* tauw, void* ustar, void* z0, int from, void* block, int block_ld,
                                 void* stream) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, output_params_t, fl3, ld, u10, udir, tauw, ustar, z0, from, block, block_ld, s);
}

int wamgpu_output_swell_dev(wamgpu_ctx* ctx, const void* fl3, int ld, const void* udir, const void* ustar, int from,
                            void* block, int block_ld, void* stream) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, output_swell_t, fl3, ld, udir, ustar, from, block, block_ld, s);
}

int wamgpu_restart_write(wamgpu_ctx* ctx, const char* path, const void* fl3, int ld, const void* u10, const void* udir,
                         const void* tauw, const void* depth, const void* u, const void* v,
                         const wamgpu_restart_dates* dates, const int* ij2newij) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  return DISPATCH_CTX(ctx, restart_write_t, path, fl3, ld, u10, udir, tauw, depth, u, v, dates, ij2newij);
}

int wamgpu_restart_read(wamgpu_ctx* ctx, const char* path, void* fl3, int ld, void* u10, void* udir, void* tauw,
                        void* depth, void* u, void* v, wamgpu_restart_dates* dates, const int* ij2newij) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  return DISPATCH_CTX(ctx, restart_read_t, path, fl3, ld, u10, udir, tauw, depth, u, v, dates, ij2newij);
}

int wamgpu_set_wind_grid(wamgpu_ctx* ctx, int nx_in, int ny_in, int west_in, int south_in, int dx_in, int dy_in,
                         int periodic, int equal_grid, int amowep, int amosop, int xdella, const int* zdello,
                         const int* ifromij) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  return DISPATCH_CTX(ctx, set_wind_grid_t, nx_in, ny_in, west_in, south_in, dx_in, dy_in, periodic, equal_grid, amowep,
                      amosop, xdella, zdello, ifromij);
}

int wamgpu_wind_dev(wamgpu_ctx* ctx, const void* u_in, const void* v_in, int code_in, void* u10, void* udir,
                    void* stream) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, wind_dev_t, u_in, v_in, code_in, u10, udir, s);
}

int wamgpu_put_points_dev(wamgpu_ctx* ctx, void* data, int ld, int nrows, const int* points, int n, double value,
                          void* stream) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, put_points_t, data, ld, nrows, points, n, value, s);
}

int wamgpu_set_diagnostics(wamgpu_ctx* ctx, int* decisions, unsigned char* llws, int ld) {
  if (!ctx) return WAMGPU_E_ARG;
  if (!decisions) { ctx->diag = nullptr; ctx->diag_ll = nullptr; ctx->diag_ld = 0; return WAMGPU_OK; }
  if (!ctx->have_grid) return fail(ctx, WAMGPU_E_STATE, "call wamgpu_set_grid first");
  if (ld < ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "diagnostics: ld < nsea");
  ctx->diag = decisions; ctx->diag_ll = llws; ctx->diag_ld = ld;
  return WAMGPU_OK;
}

int wamgpu_sync(wamgpu_ctx* ctx) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  cudaSetDevice(ctx->cfg.device);
  CK(cudaStreamSynchronize(ctx->stream), "sync");
  DevBuf* st = ctx->cfg.precision == 8 ? &static_cast<Impl<double>*>(ctx->impl.get())->status
                                       : &static_cast<Impl<float>*>(ctx->impl.get())->status;
  if (st->p) {
    int flag = 0;
    CK(cudaMemcpy(&flag, st->p, sizeof(int), cudaMemcpyDeviceToHost), "status");
    if (flag) {
      CK(cudaMemset(st->p, 0, sizeof(int)), "status");
      return fail(ctx, WAMGPU_E_NUMERIC, "non-finite values in IMPLSCH output");
    }
  }
  return WAMGPU_OK;
}

// ---- batched ensembles ---------------------------------------------------------

int wamgpu_batch_create(wamgpu_ctx* const* members, int n, wamgpu_batch** out) {
  if (!out) return WAMGPU_E_ARG;
  *out = nullptr;
  auto* b = new wamgpu_batch();
  *out = b;
  if (!members || n <= 0) return bfail(b, WAMGPU_E_ARG, "empty batch");
  for (int g = 0; g < n; ++g) {
    wamgpu_ctx* c = members[g];
    if (!c || !c->impl) return bfail(b, WAMGPU_E_ARG, "null member context");
    if (!c->prepared) return bfail(b, WAMGPU_E_STATE, "member " + std::to_string(g) + " not prepared (wamgpu_prepare_propagation)");
    if (g > 0 && (c->cfg.precision != members[0]->cfg.precision || c->cfg.device != members[0]->cfg.device))
      return bfail(b, WAMGPU_E_ARG, "members must share precision and device");
    const bool enh = c->cfg.precision == 8 ? impl_of<double>(c).has_enh : impl_of<float>(c).has_enh;
    if (c->cfg.shallow_run && c->cfg.isnonlin != 0 && !enh)
      return bfail(b, WAMGPU_E_STATE, "member " + std::to_string(g) + " needs wamgpu_prepare_source");
    b->members.push_back(c);
  }
  b->precision = members[0]->cfg.precision;
  b->device = members[0]->cfg.device;
  b->stream = members[0]->stream;
  b->st.resize(n);
  return WAMGPU_OK;
}

int wamgpu_batch_destroy(wamgpu_batch* b) {
  if (!b) return WAMGPU_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  b->drop_graph();
  delete b;
  return WAMGPU_OK;
}

const char* wamgpu_batch_last_error(const wamgpu_batch* b) { return b ? b->err.c_str() : "null batch"; }

int wamgpu_batch_set_member(wamgpu_batch* b, int g, void* fl3, int ld, void* scratch, const void* u10, const void* udir,
                            void* tauw, void* ustar, void* z0, const void* roairn, const void* wstar) {
  if (!b) return WAMGPU_E_ARG;
  if (g < 0 || g >= (int)b->members.size()) return bfail(b, WAMGPU_E_ARG, "member index out of range");
  if (!fl3 || !scratch || !u10 || !udir || !tauw || !ustar || !z0 || !roairn || !wstar) return bfail(b, WAMGPU_E_ARG, "null argument");
  if (ld < b->members[g]->nsea) return bfail(b, WAMGPU_E_ARG, "ld < nsea");
  BatchState& x = b->st[g];
  x.fl3 = fl3; x.ld = ld; x.scratch = scratch; x.u10 = u10; x.udir = udir; x.tauw = tauw; x.ustar = ustar; x.z0 = z0;
  x.roairn = roairn; x.wstar = wstar;
  b->built = false;
  b->drop_graph();
  return WAMGPU_OK;
}

int wamgpu_batch_tune(wamgpu_batch* b, void* stream, int* points_per_cta, int* propags_block) {
  if (!b) return WAMGPU_E_ARG;
  cudaSetDevice(b->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
  return b->precision == 8 ? batch_tune<double>(b, s, points_per_cta, propags_block)
                           : batch_tune<float>(b, s, points_per_cta, propags_block);
}

int wamgpu_batch_step(wamgpu_batch* b, void* stream) {
  if (!b) return WAMGPU_E_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
  if (b->exec) { BCK(cudaGraphLaunch(b->exec, s), "graph launch"); return WAMGPU_OK; }
  if (!b->built) {
    int rc = b->precision == 8 ? batch_build<double>(b, s) : batch_build<float>(b, s);
    if (rc) return rc;
  }
  return b->precision == 8 ? batch_launch<double>(b, s) : batch_launch<float>(b, s);
}

int wamgpu_batch_capture(wamgpu_batch* b, void* stream) {
  if (!b) return WAMGPU_E_ARG;
  cudaSetDevice(b->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
  b->drop_graph();
  if (!b->built) {
    int rc = b->precision == 8 ? batch_build<double>(b, s) : batch_build<float>(b, s);
    if (rc) return rc;
  }
  BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
  int rc = b->precision == 8 ? batch_launch<double>(b, s) : batch_launch<float>(b, s);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (e != cudaSuccess) return bfail(b, WAMGPU_E_CUDA, std::string("end capture: ") + cudaGetErrorString(e));
  b->graph = g;
  BCK(cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiate");
  return WAMGPU_OK;
}

int wamgpu_batch_sync(wamgpu_batch* b) {
  if (!b) return WAMGPU_E_ARG;
  cudaSetDevice(b->device);
  BCK(cudaStreamSynchronize(b->stream), "sync");
  for (size_t g = 0; g < b->members.size(); ++g) {
    int rc = wamgpu_sync(b->members[g]);
    if (rc) return bfail(b, rc, "member " + std::to_string(g) + ": " + b->members[g]->err);
  }
  return WAMGPU_OK;
}

// ---- latitude bands (one grid over several ranks) ------------------------------

int wamgpu_set_owned(wamgpu_ctx* ctx, int i0, int i1) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (!ctx->have_grid) return fail(ctx, WAMGPU_E_STATE, "set_grid first");
  if (i0 < 0 || i1 < i0 || i1 > ctx->nsea) return fail(ctx, WAMGPU_E_ARG, "owned range outside the grid");
  ctx->own0 = i0; ctx->own1 = i1;
  ctx->prepared = false;
  return WAMGPU_OK;
}

int wamgpu_set_counter(wamgpu_ctx* ctx, int counter) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  return DISPATCH_CTX(ctx, set_counter_t, counter);
}

int wamgpu_propags_substep_range_dev(wamgpu_ctx* ctx, const void* src, void* dst, int ld, int i0, int i1,
                                     void* stream) {
  if (!ctx || !ctx->impl || !src || !dst) return WAMGPU_E_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, propags_range_t, src, dst, ld, i0, i1, s);
}

int wamgpu_get_halo_width(const wamgpu_ctx* ctx) {
  if (!ctx || !ctx->have_grid) return WAMGPU_E_STATE;
  return ctx->halo;
}

int wamgpu_propags_substep_dev(wamgpu_ctx* ctx, const void* src, void* dst, int ld, void* stream) {
  if (!ctx || !ctx->impl || !src || !dst) return WAMGPU_E_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, propags_substep_t, src, dst, ld, s);
}

// ---- derivatives --------------------------------------------------------------

int wamgpu_implsch_adj_dev(wamgpu_ctx* ctx, const void* fl3_in, int ld, const void* tauw_in, const void* u10,
                           const void* udir, const void* roairn, const void* wstar, void* lam_fl3, void* lam_tauw,
                           void* lam_u10, void* stream) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (!fl3_in || !tauw_in || !u10 || !udir || !roairn || !wstar || !lam_fl3 || !lam_tauw || !lam_u10)
    return fail(ctx, WAMGPU_E_ARG, "null argument");
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, implsch_adj_t, fl3_in, ld, tauw_in, u10, udir, roairn, wstar, lam_fl3, lam_tauw, lam_u10, s);
}

int wamgpu_implsch_tl_dev(wamgpu_ctx* ctx, const void* fl3_in, const void* dfl3_in, int ld, const void* tauw_in,
                          const void* dtauw_in, const void* u10, const void* du10, const void* udir, const void* roairn,
                          const void* wstar, void* fl3_out, void* dfl3_out, void* tauw_out, void* dtauw_out,
                          void* stream) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (!fl3_in || !dfl3_in || !tauw_in || !dtauw_in || !u10 || !du10 || !udir || !roairn || !wstar || !fl3_out ||
      !dfl3_out || !tauw_out || !dtauw_out)
    return fail(ctx, WAMGPU_E_ARG, "null argument");
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, implsch_tl_t, fl3_in, dfl3_in, ld, tauw_in, dtauw_in, u10, du10, udir, roairn, wstar, fl3_out,
                      dfl3_out, tauw_out, dtauw_out, s);
}

int wamgpu_propags_adj_dev(wamgpu_ctx* ctx, void* lam_f3, int ld, void* scratch, void* stream) {
  if (!ctx || !ctx->impl || !lam_f3) return WAMGPU_E_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, propags_adj_t, lam_f3, ld, scratch, s);
}

int wamgpu_checkpoint_reserve(wamgpu_ctx* ctx, int n, int ld) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  return DISPATCH_CTX(ctx, checkpoint_reserve_t, n, ld);
}

int wamgpu_step_ckpt_dev(wamgpu_ctx* ctx, int slot, void* fl3, int ld, void* scratch, int nprop, const void* u10,
                         const void* udir, void* tauw, void* ustar, void* z0, const void* roairn, const void* wstar,
                         void* stream) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (!fl3 || !u10 || !udir || !tauw || !ustar || !z0 || !roairn || !wstar) return fail(ctx, WAMGPU_E_ARG, "null argument");
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, step_ckpt_dev_t, slot, fl3, ld, scratch, nprop, u10, udir, tauw, ustar, z0, roairn, wstar, s);
}

int wamgpu_step_adj_dev(wamgpu_ctx* ctx, int slot, int nprop, void* lam_fl3, int ld, void* lam_tauw, void* lam_u10,
                        const void* udir, const void* roairn, const void* wstar, void* scratch, void* stream) {
  if (!ctx || !ctx->impl) return WAMGPU_E_ARG;
  if (!lam_fl3 || !lam_tauw || !lam_u10 || !udir || !roairn || !wstar) return fail(ctx, WAMGPU_E_ARG, "null argument");
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  return DISPATCH_CTX(ctx, step_adj_dev_t, slot, nprop, lam_fl3, ld, lam_tauw, lam_u10, udir, roairn, wstar, scratch, s);
}

}  // extern "C"
