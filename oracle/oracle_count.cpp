// ORACLE — test infrastructure only (see oracle_tables.hpp header).
// The oracle's IMPLSCH restatement instantiated with the counting number
// type (oracle_count.hpp): floating-point operation counts of the
// reference's algorithm for given sea points.  The counting overloads of the
// <cmath> functions must be declared before the restatement's templates.
#include "oracle_count.hpp"
#include "oracle_tables.hpp"
#include "oracle_source.hpp"

using namespace wamo;

extern "C" {

// IMPLSCH (wam_source_module.f90:374-700) of nsea points with the counting
// type; counts[0..5] = additions, multiplications, divisions, square roots,
// transcendental functions, comparisons, summed over the points (the table
// preparation is not counted).  FL3(IJ,K,M) with leading dimension nsea.
int oracle_count_implsch(const OracleConfig* c, int nsea, const double* fl3, const double* u10, const double* udir,
                         const double* tauw, const double* ustar, const double* z0, const double* roairn,
                         const double* wstar, const double* depth, const int* indep, double* counts) {
  using R = CF;
  FreDir<R> fd; ShallowTables<R> sh; MinEnergy<R> me; DiaTables<R> dia; SourceTables<R> st; SourceModel<R> src;
  fd.build(c->kl, c->ml, R(c->fr1), c->iref);
  sh.build(fd, c->ndepth, R(c->deptha), R(c->depthd));
  me.build(fd, R(c->delphi));
  dia.build(fd);
  st.build(fd, c->iphys, R(c->alpha), R(c->zalp), R(c->betamax));
  src.cfg = *c; src.fd = &fd; src.sh = &sh; src.me = &me; src.dia = &dia; src.st = &st;
  src.BETAMAX = R(c->betamax); src.ZALP = R(c->zalp); src.ALPHA = R(c->alpha); src.TAUWSHELTER = R(c->tauwshelter);
  src.CDFAC = R(c->cdfac);
  if (c->shallow_run) {
    std::vector<R> d(depth, depth + nsea);
    src.make_shallow_snl(d.data(), nsea);
  }
  const int kl = c->kl, ml = c->ml;
  OpCounts tot;
  std::vector<R> F((size_t)kl * ml);
  for (int ij = 0; ij < nsea; ++ij) {
    for (int m = 0; m < ml; ++m)
      for (int k = 0; k < kl; ++k) F[k + kl * m] = R(fl3[ij + (size_t)nsea * (k + (size_t)kl * m)]);
    R tw = R(tauw[ij]), us = R(ustar[ij]), zz = R(z0[ij]);
    g_ops = OpCounts();
    src.implsch_point(F.data(), R(u10[ij]), R(udir[ij]), tw, us, zz, R(roairn[ij]), R(wstar[ij]), R(depth[ij]), indep[ij],
                      ij, nullptr);
    tot.add += g_ops.add; tot.mul += g_ops.mul; tot.div += g_ops.div; tot.sqrt += g_ops.sqrt;
    tot.trans += g_ops.trans; tot.cmp += g_ops.cmp;
  }
  counts[0] = (double)tot.add; counts[1] = (double)tot.mul; counts[2] = (double)tot.div;
  counts[3] = (double)tot.sqrt; counts[4] = (double)tot.trans; counts[5] = (double)tot.cmp;
  return 0;
}

}  // extern "C"
