// ORACLE — test infrastructure only (see oracle_tables.hpp header).
// C entry points over the restatement, loaded by tests/ and by bench.py's
// CPU-baseline leg through ctypes.  All array arguments are double precision;
// a float (REAL) oracle converts on entry and exit, which is exact for values
// that originate in single precision.
#include <cstring>
#include <string>
#include <memory>
#include <thread>
#include <atomic>
#include "oracle_tables.hpp"
#include "oracle_grid.hpp"
#include "oracle_source.hpp"
#include "oracle_prop.hpp"
#include "oracle_output.hpp"

using namespace wamo;

struct OracleBase {
  virtual ~OracleBase() {}
  int precision = 4;
};

template <typename R> struct Oracle : OracleBase {
  OracleConfig cfg;
  FreDir<R> fd; ShallowTables<R> sh; MinEnergy<R> me; DiaTables<R> dia; SourceTables<R> st;
  SourceModel<R> src; PropModel<R> prop; OutputModel<R> outm;
  std::vector<R> depth_src;  // depth of the points passed to prepare_source
  // resident REAL state of the timed CPU baseline (oracle_resident_*)
  std::vector<R> rF, rU10, rUDIR, rTAUW, rUSTAR, rZ0, rROAIRN, rWSTAR, rDEPTH;
  explicit Oracle(const OracleConfig& c) : cfg(c) {
    precision = sizeof(R);
    fd.build(c.kl, c.ml, R(c.fr1), c.iref);
    sh.build(fd, c.ndepth, R(c.deptha), R(c.depthd));
    me.build(fd, R(c.delphi));
    dia.build(fd);
    // effective module values after INITMDL's swap (initmdl.f90:153-160) are passed in
    R betamax = R(c.betamax), zalp = R(c.zalp), alpha = R(c.alpha), tauwshelter = R(c.tauwshelter);
    st.build(fd, c.iphys, alpha, zalp, betamax);
    src.cfg = c; src.fd = &fd; src.sh = &sh; src.me = &me; src.dia = &dia; src.st = &st;
    src.BETAMAX = betamax; src.ZALP = zalp; src.ALPHA = alpha; src.TAUWSHELTER = tauwshelter; src.CDFAC = R(c.cdfac);
    prop.cfg = c; prop.fd = &fd; prop.sh = &sh;
    outm.fd = &fd; outm.sh = &sh; outm.shallow = c.shallow_run != 0;
  }
};

template <typename R> static void cpy_out(const std::vector<R>& v, double* out) { for (size_t i = 0; i < v.size(); ++i) out[i] = (double)v[i]; }
template <typename R> static void cpy_out(const std::vector<int>& v, int* out) { std::memcpy(out, v.data(), v.size() * sizeof(int)); }

template <typename R> static int get_table_t(Oracle<R>* o, const std::string& n, double* out) {
  std::vector<R> tmp;
  const std::vector<R>* v = nullptr;
  if (n == "FR") v = &o->fd.FR; else if (n == "DF") v = &o->fd.DF; else if (n == "DFIM") v = &o->fd.DFIM;
  else if (n == "GOM") v = &o->fd.GOM; else if (n == "C") v = &o->fd.C; else if (n == "TH") v = &o->fd.TH;
  else if (n == "COSTH") v = &o->fd.COSTH; else if (n == "SINTH") v = &o->fd.SINTH;
  else if (n == "DFIMOFR") v = &o->fd.DFIMOFR; else if (n == "FR5") v = &o->fd.FR5; else if (n == "FRM5") v = &o->fd.FRM5;
  else if (n == "RHOWG_DFIM") v = &o->fd.RHOWG_DFIM;
  else if (n == "TFAK") v = &o->sh.TFAK; else if (n == "TCGOND") v = &o->sh.TCGOND; else if (n == "TSIHKD") v = &o->sh.TSIHKD;
  else if (n == "FLMINFR") v = &o->me.FLMINFR;
  else if (n == "AF11") v = &o->dia.AF11; else if (n == "FKLAP") v = &o->dia.FKLAP; else if (n == "FKLAP1") v = &o->dia.FKLAP1;
  else if (n == "FKLAM") v = &o->dia.FKLAM; else if (n == "FKLAM1") v = &o->dia.FKLAM1; else if (n == "FRH") v = &o->dia.FRH;
  else if (n == "RNLCOEF") v = &o->dia.RNLCOEF; else if (n == "FTRF") v = &o->dia.FTRF;
  else if (n == "SWELLFT") v = &o->st.SWELLFT; else if (n == "SATWEIGHTS") v = &o->st.SATWEIGHTS; else if (n == "WTAUHF") v = &o->st.WTAUHF;
  else if (n == "SCALARS") {
    tmp = {o->fd.DELTH, o->fd.DELTR, o->fd.INV_LOG_CO, o->fd.MO_TAIL, o->fd.MM1_TAIL, o->fd.MP1_TAIL, o->fd.MP2_TAIL,
           o->fd.FMIN, o->me.DELU, o->dia.ACL1, o->dia.ACL2, o->dia.CL11, o->dia.CL21, o->dia.DAL1, o->dia.DAL2,
           o->st.X0TAUHF, o->src.ALPHA, o->src.BETAMAX, o->src.ZALP, o->src.TAUWSHELTER, o->src.CDFAC};
    v = &tmp;
  }
  if (!v) return -1;
  if (out) cpy_out(*v, out);
  return (int)v->size();
}
template <typename R> static int get_itable_t(Oracle<R>* o, const std::string& n, int* out) {
  const std::vector<int>* v = nullptr; std::vector<int> tmp;
  if (n == "IKP") v = &o->dia.IKP; else if (n == "IKP1") v = &o->dia.IKP1; else if (n == "IKM") v = &o->dia.IKM;
  else if (n == "IKM1") v = &o->dia.IKM1; else if (n == "K1W") v = &o->dia.K1W; else if (n == "K2W") v = &o->dia.K2W;
  else if (n == "K11W") v = &o->dia.K11W; else if (n == "K21W") v = &o->dia.K21W; else if (n == "INLCOEF") v = &o->dia.INLCOEF;
  else if (n == "INDICESSAT") v = &o->st.INDICESSAT; else if (n == "MPM") v = &o->fd.MPM; else if (n == "KPM") v = &o->fd.KPM;
  else if (n == "JXO") v = &o->fd.JXO; else if (n == "JYO") v = &o->fd.JYO; else if (n == "INDEP") v = &o->prop.INDEP;
  else if (n == "DIA_SCALARS") { tmp = {o->dia.MFRSTLW, o->dia.MLSTHG, o->dia.KFRH, o->dia.ISP, o->dia.ISM, o->st.NSDSNTH}; v = &tmp; }
  else if (n == "COUNTER") { tmp = {o->prop.COUNTER}; v = &tmp; }
  if (!v) return -1;
  if (out) std::memcpy(out, v->data(), v->size() * sizeof(int));
  return (int)v->size();
}

template <typename R> static void implsch_t(Oracle<R>* o, int nsea, int ld, double* fl3, const double* u10, const double* udir,
                                            double* tauw, double* ustar, double* z0, const double* roairn, const double* wstar,
                                            const double* depth, const int* indep, double* fluxes, int nthreads,
                                            int* idiag = nullptr, double* fdiag = nullptr, unsigned char* llws = nullptr) {
  const int kl = o->fd.KL, ml = o->fd.ML;
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::atomic<int> next(0);
  auto work = [&]() {
  for (;;) {
    int ij = next.fetch_add(1);
    if (ij >= nsea) break;
    std::vector<R> F((size_t)kl * ml);
    for (int m = 0; m < ml; ++m)
      for (int k = 0; k < kl; ++k) F[k + kl * m] = R(fl3[ij + (size_t)ld * (k + (size_t)kl * m)]);
    R tw = R(tauw[ij]), us = R(ustar[ij]), zz = R(z0[ij]);
    typename SourceModel<R>::Fluxes fx{};
    typename SourceModel<R>::Diag dg{};
    std::vector<uint8_t> m1, m2;
    if (llws) { m1.resize((size_t)kl * ml); m2.resize((size_t)kl * ml); dg.LLWS1 = m1.data(); dg.LLWS2 = m2.data(); }
    o->src.implsch_point(F.data(), R(u10[ij]), R(udir[ij]), tw, us, zz, R(roairn[ij]), R(wstar[ij]), R(depth[ij]), indep[ij],
                         ij, fluxes ? &fx : nullptr, (idiag || fdiag || llws) ? &dg : nullptr);
    if (idiag) { idiag[ij] = dg.JU; idiag[ij + nsea] = dg.MIJ1; idiag[ij + 2 * (size_t)nsea] = dg.MIJ2; idiag[ij + 3 * (size_t)nsea] = dg.LFIT; }
    if (fdiag) {
      fdiag[ij] = dg.JU_ARG; fdiag[ij + nsea] = dg.MIJ1_ARG; fdiag[ij + 2 * (size_t)nsea] = dg.MIJ2_ARG;
      fdiag[ij + 3 * (size_t)nsea] = dg.LF_MARGIN;
    }
    if (llws) {
      const size_t ns = (size_t)kl * ml;
      for (size_t b = 0; b < ns; ++b) { llws[ij + nsea * b] = m1[b]; llws[ij + nsea * (b + ns)] = m2[b]; }
    }
    for (int m = 0; m < ml; ++m)
      for (int k = 0; k < kl; ++k) fl3[ij + (size_t)ld * (k + (size_t)kl * m)] = (double)F[k + kl * m];
    tauw[ij] = tw; ustar[ij] = us; z0[ij] = zz;
    if (fluxes) {
      R v[7] = {fx.PHIOC, fx.TAUOC_X, fx.TAUOC_Y, fx.PHIBOT, fx.TAUBOT_X, fx.TAUBOT_Y, fx.PHIAW};
      for (int i = 0; i < 7; ++i) fluxes[ij + (size_t)nsea * i] = (double)v[i];
    }
  }
  };
  if (nthreads == 1) { work(); return; }
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t) pool.emplace_back(work);
  for (auto& t : pool) t.join();
}

// One WAMODEL pass (wamodel.f90:286-360) on the resident state: nprop
// PROPAGS calls, then IMPLSCH over every sea point, with nthreads host
// threads (planes of PROPAGS, sea points of IMPLSCH) and no conversions.
template <typename R> static void resident_step_t(Oracle<R>* o, int nprop, int nthreads) {
  const int kl = o->fd.KL, ml = o->fd.ML, nsea = o->prop.NSEA;
  R* FL3 = o->rF.data();
  for (int p = 0; p < nprop; ++p) o->prop.propags(FL3, nthreads);
  const int* indep = &o->prop.INDEP[1];
  std::atomic<int> next(0);
  auto work = [&]() {
    std::vector<R> F((size_t)kl * ml);
    for (int ij; (ij = next.fetch_add(1)) < nsea;) {
      for (int m = 0; m < ml; ++m)
        for (int k = 0; k < kl; ++k) F[k + kl * m] = FL3[ij + (size_t)nsea * (k + (size_t)kl * m)];
      o->src.implsch_point(F.data(), o->rU10[ij], o->rUDIR[ij], o->rTAUW[ij], o->rUSTAR[ij], o->rZ0[ij], o->rROAIRN[ij],
                           o->rWSTAR[ij], o->rDEPTH[ij], indep[ij], ij, nullptr);
      for (int m = 0; m < ml; ++m)
        for (int k = 0; k < kl; ++k) FL3[ij + (size_t)nsea * (k + (size_t)kl * m)] = F[k + kl * m];
    }
  };
  if (nthreads <= 1) { work(); return; }
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t) pool.emplace_back(work);
  for (auto& t : pool) t.join();
}

extern "C" {

void* oracle_create(const OracleConfig* cfg, int precision) {
  try {
    if (precision == 8) return new Oracle<double>(*cfg);
    return new Oracle<float>(*cfg);
  } catch (...) { return nullptr; }
}
void oracle_destroy(void* h) { delete (OracleBase*)h; }

#define DISPATCH(h, call) \
  (((OracleBase*)(h))->precision == 8 ? (call((Oracle<double>*)(h))) : (call((Oracle<float>*)(h))))

// Resident state for the timed CPU baseline: FL3(IJ,K,M) of NSEA points and
// the per-point fields, converted once to the oracle's precision.
int oracle_resident_set(void* h, const double* fl3, const double* u10, const double* udir, const double* tauw,
                        const double* ustar, const double* z0, const double* roairn, const double* wstar,
                        const double* depth) {
  auto f = [&](auto* o) {
    using RR = typename std::decay<decltype(o->fd.FR[0])>::type;
    const size_t n = (size_t)o->prop.NSEA, nb = n * o->fd.KL * o->fd.ML;
    auto cv = [](const double* a, size_t m) { std::vector<RR> v(m); for (size_t i = 0; i < m; ++i) v[i] = RR(a[i]); return v; };
    o->rF = cv(fl3, nb); o->rU10 = cv(u10, n); o->rUDIR = cv(udir, n); o->rTAUW = cv(tauw, n); o->rUSTAR = cv(ustar, n);
    o->rZ0 = cv(z0, n); o->rROAIRN = cv(roairn, n); o->rWSTAR = cv(wstar, n); o->rDEPTH = cv(depth, n);
    return 0;
  };
  return DISPATCH(h, f);
}
int oracle_resident_step(void* h, int nprop, int nthreads) {
  auto f = [&](auto* o) {
    if (o->rF.size() != (size_t)o->prop.NSEA * o->fd.KL * o->fd.ML) return -1;
    resident_step_t(o, nprop, nthreads);
    return 0;
  };
  return DISPATCH(h, f);
}
int oracle_resident_get(void* h, double* fl3, double* tauw, double* ustar, double* z0) {
  auto f = [&](auto* o) {
    for (size_t i = 0; i < o->rF.size(); ++i) fl3[i] = (double)o->rF[i];
    for (size_t i = 0; i < o->rTAUW.size(); ++i) { tauw[i] = o->rTAUW[i]; ustar[i] = o->rUSTAR[i]; z0[i] = o->rZ0[i]; }
    return 0;
  };
  return DISPATCH(h, f);
}

// COMPUTE_OUTPUT_PARAMETER (wam_output_module.f90:481-640) for nsea points:
// out[ij + nsea*(IP-1)], IP = 1..40 (parameters not restated stay 0).
// ustar and z0 are in/out: AIRSEA sets them when USTAR is zero everywhere.
int oracle_output_params(void* h, int nsea, const double* fl3, const double* u10, const double* udir, double* ustar,
                         const double* tauw, double* z0, const double* depth, const double* u, const double* v,
                         const int* indep, int from, double* out) {
  auto f = [&](auto* o) {
    using RR = typename std::decay<decltype(o->fd.FR[0])>::type;
    const int kl = o->fd.KL, ml = o->fd.ML;
    double mx = 0;
    for (int i = 0; i < nsea; ++i) mx = std::max(mx, ustar[i]);
    o->outm.from = from != 0;
    std::vector<RR> F((size_t)kl * ml), P(OUT_NPARAM);
    for (int ij = 0; ij < nsea; ++ij) {
      for (int m = 0; m < ml; ++m)
        for (int k = 0; k < kl; ++k) F[k + kl * m] = RR(fl3[ij + (size_t)nsea * (k + (size_t)kl * m)]);
      RR us = RR(ustar[ij]), zz = RR(z0[ij]);
      if (mx == 0) { o->src.airsea(RR(u10[ij]), RR(tauw[ij]), us, zz); ustar[ij] = us; z0[ij] = zz; }
      o->outm.point(F.data(), RR(u10[ij]), RR(udir[ij]), us, RR(tauw[ij]), zz, RR(depth[ij]), u ? RR(u[ij]) : RR(0),
                    v ? RR(v[ij]) : RR(0), indep[ij], P.data());
      for (int p = 0; p < OUT_NPARAM; ++p) out[ij + (size_t)nsea * p] = (double)P[p];
    }
    return 0;
  };
  return DISPATCH(h, f);
}

// SWELL_SEPARATION (wam_swell_module.f90:106-350) for nsea points:
// out[ij + nsea*(IP-1)] for IP = 17..23 and 25..31 (the other rows untouched).
int oracle_output_swell(void* h, int nsea, const double* fl3, const double* udir, const double* ustar, int from,
                        double* out) {
  auto f = [&](auto* o) {
    using RR = typename std::decay<decltype(o->fd.FR[0])>::type;
    const int kl = o->fd.KL, ml = o->fd.ML;
    o->outm.from = from != 0;
    std::vector<RR> F((size_t)kl * ml), P(OUT_NPARAM, RR(0));
    for (int ij = 0; ij < nsea; ++ij) {
      for (int m = 0; m < ml; ++m)
        for (int k = 0; k < kl; ++k) F[k + kl * m] = RR(fl3[ij + (size_t)nsea * (k + (size_t)kl * m)]);
      o->outm.swell(F.data(), RR(udir[ij]), RR(ustar[ij]), P.data());
      for (int p = 17; p <= 31; ++p)
        if (p != 24) out[ij + (size_t)nsea * (p - 1)] = (double)P[p - 1];
    }
    return 0;
  };
  return DISPATCH(h, f);
}

int oracle_get_table(void* h, const char* name, double* out) {
  std::string n(name);
  auto f = [&](auto* o) { return get_table_t(o, n, out); };
  return DISPATCH(h, f);
}
int oracle_get_itable(void* h, const char* name, int* out) {
  std::string n(name);
  auto f = [&](auto* o) { return get_itable_t(o, n, out); };
  return DISPATCH(h, f);
}

int oracle_set_grid(void* h, int nsea, const int* klat, const int* klon, const double* wlat, const int* kfromij, int ny,
                    const double* sinph, const double* cosph, const double* dellam, double delphi) {
  if (((OracleBase*)h)->precision == 8) {
    auto* o = (Oracle<double>*)h;
    std::vector<double> w(wlat, wlat + (size_t)nsea * 2);
    o->prop.set_grid(nsea, klat, klon, w.data(), kfromij, ny, sinph, cosph, dellam, delphi);
  } else {
    auto* o = (Oracle<float>*)h;
    std::vector<float> w(wlat, wlat + (size_t)nsea * 2), s(sinph, sinph + ny), c(cosph, cosph + ny), d(dellam, dellam + ny);
    o->prop.set_grid(nsea, klat, klon, w.data(), kfromij, ny, s.data(), c.data(), d.data(), (float)delphi);
  }
  return 0;
}

int oracle_set_fields(void* h, const double* depth, const double* u, const double* v) {
  auto f = [&](auto* o) {
    using RR = typename std::decay<decltype(o->fd.FR[0])>::type;
    int n = o->prop.NSEA;
    std::vector<RR> d(n), uu(n, RR(0)), vv(n, RR(0));
    for (int i = 0; i < n; ++i) { d[i] = RR(depth[i]); if (u) uu[i] = RR(u[i]); if (v) vv[i] = RR(v[i]); }
    o->prop.set_depth(d.data()); o->prop.set_current(uu.data(), vv.data());
    o->depth_src = d;
    return 0;
  };
  return DISPATCH(h, f);
}

int oracle_prepare_propagation(void* h, double* cfl, int* counter) {
  auto f = [&](auto* o) {
    int rc = o->prop.prepare();
    if (cfl) *cfl = (double)o->prop.total_cfl;
    if (counter) *counter = o->prop.COUNTER;
    return rc;
  };
  return DISPATCH(h, f);
}

int oracle_prepare_source(void* h) {
  auto f = [&](auto* o) {
    if (o->cfg.shallow_run) o->src.make_shallow_snl(o->depth_src.data(), (int)o->depth_src.size());
    return 0;
  };
  return DISPATCH(h, f);
}

// Sea-point depth-table index INDEP (PREPARE_PROPAGATION :327-332).
int oracle_get_indep(void* h, int* out) {
  auto f = [&](auto* o) { for (int i = 0; i < o->prop.NSEA; ++i) out[i] = o->prop.INDEP[i + 1]; return o->prop.NSEA; };
  return DISPATCH(h, f);
}

int oracle_get_coef(void* h, const char* name, double* out) {
  std::string n(name);
  auto f = [&](auto* o) {
    const auto* v = &o->prop.COEF_SUM;
    if (n == "LAT") v = &o->prop.COEF_LAT; else if (n == "LON") v = &o->prop.COEF_LON;
    else if (n == "THETA") v = &o->prop.COEF_THETA; else if (n == "SIGD") v = &o->prop.COEF_SIGD;
    if (out) for (size_t i = 0; i < v->size(); ++i) out[i] = (double)(*v)[i];
    return (int)v->size();
  };
  return DISPATCH(h, f);
}

// One IMPLSCH call on nsea points.  fl3 is FL3(IJ,K,M) with leading dimension
// ld >= nsea.  fluxes (optional, LCFLX) receives PHIOC, TAUOC_X, TAUOC_Y,
// PHIBOT, TAUBOT_X, TAUBOT_Y, PHIAW as 7 blocks of nsea.
int oracle_implsch(void* h, int nsea, int ld, double* fl3, const double* u10, const double* udir, double* tauw, double* ustar,
                   double* z0, const double* roairn, const double* wstar, const double* depth, const int* indep,
                   double* fluxes, int nthreads) {
  auto f = [&](auto* o) {
    implsch_t(o, nsea, ld, fl3, u10, udir, tauw, ustar, z0, roairn, wstar, depth, indep, fluxes, nthreads);
    return 0;
  };
  return DISPATCH(h, f);
}

// oracle_implsch that also returns the step's integer decisions: idiag
// (4 blocks of nsea: JU, MIJ of the first and of the last FRCUTINDEX call,
// LFACTOR iterations), fdiag (the REAL values they were rounded from, and
// the smallest relative distance of the LFACTOR |ERR| from its exit threshold) and llws (2 planes of KL*ML blocks of nsea: the
// LLWS masks of the first and of the last SINPUT call), each optional.
int oracle_implsch_diag(void* h, int nsea, int ld, double* fl3, const double* u10, const double* udir, double* tauw,
                        double* ustar, double* z0, const double* roairn, const double* wstar, const double* depth,
                        const int* indep, double* fluxes, int nthreads, int* idiag, double* fdiag, unsigned char* llws) {
  auto f = [&](auto* o) {
    implsch_t(o, nsea, ld, fl3, u10, udir, tauw, ustar, z0, roairn, wstar, depth, indep, fluxes, nthreads, idiag, fdiag,
              llws);
    return 0;
  };
  return DISPATCH(h, f);
}

// One PROPAGS call (COUNTER sub-steps) on F3(IJ,K,M), leading dimension NSEA.
int oracle_propags(void* h, double* f3) {
  auto f = [&](auto* o) {
    using RR = typename std::decay<decltype(o->fd.FR[0])>::type;
    size_t n = (size_t)o->prop.NSEA * o->fd.KL * o->fd.ML;
    std::vector<RR> F(n);
    for (size_t i = 0; i < n; ++i) F[i] = RR(f3[i]);
    o->prop.propags(F.data(), (int)std::max(1u, std::thread::hardware_concurrency()));
    for (size_t i = 0; i < n; ++i) f3[i] = (double)F[i];
    return 0;
  };
  return DISPATCH(h, f);
}

// ---- grid builder (REAL precision, as the reference preprocessor) ------------
void* oracle_grid_create(const GridDef* g, const unsigned char* mask) {
  auto* gr = new Grid<float>();
  std::vector<uint8_t> mk(mask, mask + (size_t)g->NX * g->NY);
  gr->build(*g, mk);
  return gr;
}
void oracle_grid_destroy(void* h) { delete (Grid<float>*)h; }
int oracle_grid_nsea(void* h) { return ((Grid<float>*)h)->NSEA; }
int oracle_grid_get(void* h, int* klat, int* klon, double* wlat, int* kfromij, double* sinph, double* cosph, double* dellam,
                    double* delphi, int* ixlg, int* kxlt, int* iper) {
  auto* g = (Grid<float>*)h;
  std::memcpy(klat, g->KLAT.data(), g->KLAT.size() * sizeof(int));
  std::memcpy(klon, g->KLON.data(), g->KLON.size() * sizeof(int));
  for (size_t i = 0; i < g->WLAT.size(); ++i) wlat[i] = g->WLAT[i];
  std::memcpy(kfromij, g->KFROMIJ.data(), g->KFROMIJ.size() * sizeof(int));
  for (int k = 0; k < g->NY; ++k) { sinph[k] = g->SINPH[k]; cosph[k] = g->COSPH[k]; dellam[k] = g->DELLAM[k]; }
  *delphi = g->DELPHI;
  std::memcpy(ixlg, g->IXLG.data(), g->IXLG.size() * sizeof(int));
  std::memcpy(kxlt, g->KXLT.data(), g->KXLT.size() * sizeof(int));
  *iper = g->IPER ? 1 : 0;
  return g->NSEA;
}

int oracle_sizeof_config() { return (int)sizeof(OracleConfig); }
int oracle_sizeof_griddef() { return (int)sizeof(GridDef); }

}  // extern "C"
