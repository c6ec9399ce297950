// Adjoint (one sea point per warp, work arrays in shared memory; ST4 and ST6)
// and tangent-linear (one sea point per thread, work arrays in global memory
// with the sea point fastest; ST4) kernels of IMPLSCH.
#include <mutex>
#include "adjoint_warp.cuh"
#include "kernels.hpp"

namespace wamgpu {

template <typename R> __device__ __forceinline__ adj::PointIn<R> point_in(const DerivArgs<R>& a, int ij) {
  adj::PointIn<R> P;
  P.INDEP = a.indep[ij]; P.DEPTH = a.depth[ij]; P.UDIR = a.udir[ij]; P.ROAIRN = a.roairn[ij]; P.WSTAR = a.wstar[ij];
  P.ENH.p = a.enh ? a.enh + ij : nullptr;
  P.ENH.ld = (size_t)a.enh_ld;
  return P;
}

// The source tables as the dual-number routines see them: scalars from the
// kernel parameter, arrays in the CTA's shared-memory copy.
template <typename R> __device__ adj::ATabs<R> atabs_view(const DevTables<R>& T, const STabs<R>& S) {
  adj::ATabs<R> A;
  A.KL = T.KL; A.ML = T.ML; A.NDEPTH = T.NDEPTH; A.MFRSTLW = T.MFRSTLW; A.MLSTHG = T.MLSTHG; A.KFRH = T.KFRH;
  A.NSDSNTH = T.NSDSNTH; A.shallow = T.shallow; A.isnonlin = T.isnonlin;
  A.DELTH = T.DELTH; A.INV_LOG_CO = T.INV_LOG_CO; A.MO_TAIL = T.MO_TAIL; A.MM1_TAIL = T.MM1_TAIL; A.DELU = T.DELU;
  A.DAL1 = T.DAL1; A.DAL2 = T.DAL2; A.X0TAUHF = T.X0TAUHF; A.BETAMAX = T.BETAMAX; A.ZALP = T.ZALP; A.ALPHA = T.ALPHA;
  A.TAUWSHELTER = T.TAUWSHELTER; A.DELT = T.DELT;
  A.FR = S.FR; A.DFIM = S.DFIM; A.DFIMOFR = S.DFIMOFR; A.FR5 = S.FR5; A.FRM5 = S.FRM5; A.RHOWG = S.RHOWG; A.TH = S.TH;
  A.COSTH = S.COSTH; A.SINTH = S.SINTH; A.DELFL = S.DELFL; A.AF11 = S.AF11; A.RNL = S.RNL; A.SATW = S.SATW;
  A.WTAUHF = S.WTAUHF; A.SWELLFT = S.SWELLFT; A.TFAK = T.TFAK; A.TCGOND = T.TCGOND; A.FLMINFR = T.FLMINFR;
  A.K1W = S.K1W; A.K2W = S.K2W; A.K11W = S.K11W; A.K21W = S.K21W; A.INL = S.INL; A.IKP = S.IKP; A.IKP1 = S.IKP1;
  A.IKM = S.IKM; A.IKM1 = S.IKM1; A.INDSAT = S.INDSAT;
  return A;
}

// CTA of P warps = P consecutive sea points.  The spectra and their adjoints
// are staged into shared memory with consecutive threads on consecutive
// points of one bin, and the adjoints written back the same way.  The warps
// of a CTA pass the phases of the step together (a CTA barrier after each):
// the step's code is far larger than the instruction cache, and warps in
// different phases would keep evicting each other's code.  A warp beyond the
// last sea point repeats the last point and writes nothing.
template <typename R, int P>
__global__ void __launch_bounds__(P * 32) implsch_adj_kernel(const __grid_constant__ DevTables<R> T,
                                                             const __grid_constant__ DerivArgs<R> a) {
  extern __shared__ __align__(16) unsigned char smem[];
  R* sR = reinterpret_cast<R*>(smem);
  int* sI = reinterpret_cast<int*>(sR + T.lay.nreal);
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int i = tid; i < T.lay.nreal; i += nthr) sR[i] = T.small[i];
  for (int i = tid; i < T.lay.nint; i += nthr) sI[i] = T.ismall[i];
  const int NS = T.NS, KL = T.KL, LD = T.ld, ML = T.ML;
  const size_t wsb = adjw_ws_bytes<R>(LD, ML, T.scr);
  unsigned char* ws0 = smem + tables_bytes<R>(T.lay);
  const size_t foff = ws_f_offset<R>(LD, ML), loff = adjw_lam_offset<R>(LD, ML, T.scr);
  const int ij0 = blockIdx.x * P;
  const size_t ld = (size_t)a.ld;
  // stage F and its adjoint with cp.async: thread t takes point t mod P and
  // bins t div P + 32 j, whose (m, k) advance by a carry
  const int tp = tid % P, tb = tid / P, dq = 32 / KL, dr = 32 - dq * KL;
  {
    const int ij = min(ij0 + tp, a.nsea - 1);
    unsigned char* base = ws0 + tp * wsb;
    R* dF = reinterpret_cast<R*>(base + foff);
    R* dL = reinterpret_cast<R*>(base + loff);
    int m = tb / KL, k = tb - m * KL;
    for (int b = tb; b < NS; b += 32) {
      const unsigned sf = (unsigned)__cvta_generic_to_shared(dF + k + LD * m);
      const unsigned sl = (unsigned)__cvta_generic_to_shared(dL + k + LD * m);
      const R* gf = a.fl3_in + ij + ld * b;
      const R* gl = a.lam_fl3 + ij + ld * b;
      if (sizeof(R) == 4) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sf), "l"(gf) : "memory");
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sl), "l"(gl) : "memory");
      } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sf), "l"(gf) : "memory");
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sl), "l"(gl) : "memory");
      }
      k += dr; m += dq;
      if (k >= KL) { k -= KL; ++m; }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, ij = min(ij0 + warp, a.nsea - 1);
  {
    STabs<R> S;
    S.bind(sR, sI, T.lay);
    WarpWS<R> w;
    unsigned char* base = ws0 + warp * wsb;
    w.ld = LD; w.scr = T.scr;
    w.SF = reinterpret_cast<typename WarpWS<R>::R2*>(base);
    w.F = reinterpret_cast<R*>(base + foff);
    w.SP = nullptr;
    w.T = reinterpret_cast<R*>(base + ws_t_offset<R>(LD, ML, 0));
    w.LL = reinterpret_cast<uint8_t*>(w.T + 8 * T.scr);
    Src<R> src(T, S, w, lane, ij, a.indep[ij], a.u10[ij], a.udir[ij], a.roairn[ij], a.wstar[ij], a.depth[ij], a.enh,
               a.enh_ld);
    if (a.lfin) src.lfreplay = a.lfin + ij;
    const adj::ATabs<R> A = atabs_view(T, S);
    adj::PointIn<R> pin;
    pin.INDEP = a.indep[ij]; pin.DEPTH = a.depth[ij]; pin.UDIR = a.udir[ij]; pin.ROAIRN = a.roairn[ij];
    pin.WSTAR = a.wstar[ij];
    pin.ENH.p = a.enh ? a.enh + ij : nullptr;
    pin.ENH.ld = (size_t)a.enh_ld;
    AdjW<R> g(src, A, pin, a.fl3_in + ij, ld, reinterpret_cast<R*>(base + loff),
              reinterpret_cast<R*>(base + adjw_at_offset<R>(LD, ML, T.scr)), base + adjw_ll1_offset<R>(LD, ML, T.scr));
    const R tw0 = a.tauw_in[ij], ltw = a.lam_tauw[ij];
    R lT0 = 0, lU = 0;
    if (T.iphys == 2) {
      g.forward6();
      g.reverse6(ltw, lT0, lU);
    } else {
      g.forward(tw0);
      g.reverse(tw0, ltw, lT0, lU);
    }
    if (lane == 0 && ij0 + warp < a.nsea) { a.lam_tauw[ij] = lT0; a.lam_u10[ij] = lU; }
  }
  __syncthreads();
  R* lout = a.lam_out ? a.lam_out : a.lam_fl3;
  if (ij0 + tp < a.nsea) {
    const R* sL = reinterpret_cast<const R*>(ws0 + tp * wsb + loff);
    R* dst = lout + ij0 + tp;
    int m = tb / KL, k = tb - m * KL;
    for (int b = tb; b < NS; b += 32) {
      dst[ld * b] = sL[k + LD * m];
      k += dr; m += dq;
      if (k >= KL) { k -= KL; ++m; }
    }
  }
}

template <typename R> size_t adj_smem_bytes(const DevTables<R>& T, int P) {
  return tables_bytes<R>(T.lay) + (size_t)P * adjw_ws_bytes<R>(T.ld, T.ML, T.scr);
}

// Raise-only opt-in shared-memory limit per instance (process state of the device).
template <typename R, int P> cudaError_t adj_set_smem(size_t bytes) {
  static std::mutex mu;
  static size_t cur[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(mu);
  if (bytes <= cur[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute(implsch_adj_kernel<R, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur[dev] = bytes;
  return e;
}

template <typename R, int P>
cudaError_t adj_launch_one(const DevTables<R>& T, const DerivArgs<R>& a, int ctas, cudaStream_t s) {
  const size_t bytes = adj_smem_bytes(T, P);
  cudaError_t e = adj_set_smem<R, P>(bytes);
  if (e != cudaSuccess) return e;
  (void)ctas;
  implsch_adj_kernel<R, P><<<(a.nsea + P - 1) / P, P * 32, bytes, s>>>(T, a);
  return cudaGetLastError();
}

// Sea points per CTA: the compiled shape that keeps the most warps resident
// per SM under the shared-memory budget (ties go to smaller CTAs); `ctas`
// receives the number of resident CTAs over the device.
template <typename R> int adj_points_per_cta(const DevTables<R>& T, int dev, int& ctas) {
  int optin = 0, persm = 0, nsm = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&persm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  const int cand32[] = {2, 4, 6, 8, 9}, cand64[] = {1, 2, 3, 4, 5};
  const int* cand = sizeof(R) == 4 ? cand32 : cand64;
  const int nc = 5;
  int best = 0, best_warps = 0;
  for (int i = 0; i < nc; ++i) {
    const size_t b = adj_smem_bytes(T, cand[i]);
    if (b > (size_t)optin) continue;
    const int per = (int)(persm / (b + 1024)), warps = cand[i] * per;
    if (warps > best_warps) { best = cand[i]; best_warps = warps; ctas = per * nsm; }
  }
  return best;
}

template <typename R> cudaError_t launch_implsch_adj(const DevTables<R>& T, const DerivArgs<R>& a, cudaStream_t s) {
  if (a.nsea == 0) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int ctas = 0;
  const int P = adj_points_per_cta(T, dev, ctas);
  if constexpr (sizeof(R) == 4) {
    if (P == 9) return adj_launch_one<R, 9>(T, a, ctas, s);
    if (P == 8) return adj_launch_one<R, 8>(T, a, ctas, s);
    if (P == 6) return adj_launch_one<R, 6>(T, a, ctas, s);
    if (P == 4) return adj_launch_one<R, 4>(T, a, ctas, s);
    if (P == 2) return adj_launch_one<R, 2>(T, a, ctas, s);
  } else {
    if (P == 5) return adj_launch_one<R, 5>(T, a, ctas, s);
    if (P == 4) return adj_launch_one<R, 4>(T, a, ctas, s);
    if (P == 3) return adj_launch_one<R, 3>(T, a, ctas, s);
    if (P == 2) return adj_launch_one<R, 2>(T, a, ctas, s);
    if (P == 1) return adj_launch_one<R, 1>(T, a, ctas, s);
  }
  return cudaErrorInvalidConfiguration;  // one point's work arrays exceed the shared memory of a CTA
}

template <typename R>
__global__ void __launch_bounds__(128) implsch_tl_kernel(const __grid_constant__ DerivArgs<R> a) {
  const int ij = blockIdx.x * blockDim.x + threadIdx.x;
  if (ij >= a.nsea) return;
  using namespace adj;
  using D = Dual<R>;
  const int nb = a.A.KL * a.A.ML;
  const size_t ls = (size_t)a.ld, lw = (size_t)a.nsea;
  D* w = reinterpret_cast<D*>(a.work) + ij;
  uint8_t* mk = a.masks + ij;
  const PointIn<R> P = point_in(a, ij);
  Col<D> f0{w + lw * 4 * nb, lw};
  for (int b = 0; b < nb; ++b) f0[b] = D(a.fl3_in[ij + ls * b], a.dfl3_in[ij + ls * b]);
  int it[TI_COUNT];
  D tw, us, z0;
  forward<R, D>(a.A, P, Col<const D>{f0.p, lw}, D(a.tauw_in[ij], a.dtauw_in[ij]), D(a.u10[ij], a.du10[ij]),
                Col<D>{w, lw}, Col<D>{w + lw * nb, lw}, Col<D>{w + lw * 2 * nb, lw}, Col<uint8_t>{mk, lw},
                Col<uint8_t>{mk + lw * nb, lw}, Col<D>{w + lw * 5 * nb, lw}, it, tw, us, z0);
  for (int b = 0; b < nb; ++b) {
    const D v = w[lw * b];
    a.fl3_out[ij + ls * b] = v.v;
    a.dfl3_out[ij + ls * b] = v.d;
  }
  a.tauw_out[ij] = tw.v; a.dtauw_out[ij] = tw.d;
  if (a.ustar_out) a.ustar_out[ij] = us.v;
  if (a.z0_out) a.z0_out[ij] = z0.v;
}

// Global work bytes per sea point of the tangent-linear kernel.
template <typename R> size_t deriv_work_bytes(int KL, int ML) {
  const size_t nb = (size_t)KL * ML, tp = (size_t)adj::tape_size(ML);
  return (5 * nb + tp) * sizeof(adj::Dual<R>);
}

template <typename R> cudaError_t launch_implsch_tl(const DerivArgs<R>& a, cudaStream_t s) {
  if (a.nsea == 0) return cudaSuccess;
  implsch_tl_kernel<R><<<(a.nsea + 127) / 128, 128, 0, s>>>(a);
  return cudaGetLastError();
}

template size_t deriv_work_bytes<float>(int, int);
template size_t deriv_work_bytes<double>(int, int);
template cudaError_t launch_implsch_adj<float>(const DevTables<float>&, const DerivArgs<float>&, cudaStream_t);
template cudaError_t launch_implsch_adj<double>(const DevTables<double>&, const DerivArgs<double>&, cudaStream_t);
template cudaError_t launch_implsch_tl<float>(const DerivArgs<float>&, cudaStream_t);
template cudaError_t launch_implsch_tl<double>(const DerivArgs<double>&, cudaStream_t);

}  // namespace wamgpu
