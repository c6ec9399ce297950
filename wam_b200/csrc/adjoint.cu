// Tangent-linear and adjoint kernels of IMPLSCH (ST4): one sea point per
// thread, per-point work arrays in global memory with the sea point fastest.
#include "adjoint.cuh"
#include "kernels.hpp"

namespace wamgpu {

template <typename R> __device__ __forceinline__ adj::PointIn<R> point_in(const DerivArgs<R>& a, int ij) {
  adj::PointIn<R> P;
  P.INDEP = a.indep[ij]; P.DEPTH = a.depth[ij]; P.UDIR = a.udir[ij]; P.ROAIRN = a.roairn[ij]; P.WSTAR = a.wstar[ij];
  P.ENH.p = a.enh ? a.enh + ij : nullptr;
  P.ENH.ld = (size_t)a.enh_ld;
  return P;
}

template <typename R>
__global__ void __launch_bounds__(128) implsch_adj_kernel(const __grid_constant__ DerivArgs<R> a) {
  const int ij = blockIdx.x * blockDim.x + threadIdx.x;
  if (ij >= a.nsea) return;
  using namespace adj;
  const int nb = a.A.KL * a.A.ML;
  const size_t ls = (size_t)a.ld, lw = (size_t)a.nsea;
  R* w = reinterpret_cast<R*>(a.work) + ij;
  uint8_t* mk = a.masks + ij;
  const PointIn<R> P = point_in(a, ij);
  R lT0 = 0, lU = 0;
  reverse<R>(a.A, P, Col<const R>{a.fl3_in + ij, ls}, a.tauw_in[ij], a.u10[ij], Col<R>{w, lw}, Col<R>{w + lw * nb, lw},
             Col<R>{w + lw * 2 * nb, lw}, Col<uint8_t>{mk, lw}, Col<uint8_t>{mk + lw * nb, lw},
             Col<R>{w + lw * 5 * nb, lw}, Col<R>{a.lam_fl3 + ij, ls}, Col<R>{w + lw * 3 * nb, lw},
             Col<R>{w + lw * 4 * nb, lw}, a.lam_tauw[ij], lT0, lU);
  a.lam_tauw[ij] = lT0;
  a.lam_u10[ij] = lU;
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

// Work bytes per sea point of the two kernels.
template <typename R> size_t deriv_work_bytes(int KL, int ML, bool tl) {
  const size_t nb = (size_t)KL * ML, tp = (size_t)adj::tape_size(ML);
  return tl ? (5 * nb + tp) * sizeof(adj::Dual<R>) : (5 * nb + tp) * sizeof(R);
}

template <typename R> cudaError_t launch_implsch_adj(const DerivArgs<R>& a, cudaStream_t s) {
  if (a.nsea == 0) return cudaSuccess;
  implsch_adj_kernel<R><<<(a.nsea + 127) / 128, 128, 0, s>>>(a);
  return cudaGetLastError();
}
template <typename R> cudaError_t launch_implsch_tl(const DerivArgs<R>& a, cudaStream_t s) {
  if (a.nsea == 0) return cudaSuccess;
  implsch_tl_kernel<R><<<(a.nsea + 127) / 128, 128, 0, s>>>(a);
  return cudaGetLastError();
}

template size_t deriv_work_bytes<float>(int, int, bool);
template size_t deriv_work_bytes<double>(int, int, bool);
template cudaError_t launch_implsch_adj<float>(const DerivArgs<float>&, cudaStream_t);
template cudaError_t launch_implsch_adj<double>(const DerivArgs<double>&, cudaStream_t);
template cudaError_t launch_implsch_tl<float>(const DerivArgs<float>&, cudaStream_t);
template cudaError_t launch_implsch_tl<double>(const DerivArgs<double>&, cudaStream_t);

}  // namespace wamgpu
