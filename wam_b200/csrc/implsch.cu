// IMPLSCH kernel entry: CTA of P warps = P consecutive sea points.
#include "implsch.cuh"
#include "kernels.hpp"

namespace wamgpu {

template <typename R>
__host__ __device__ inline size_t tables_bytes(const SmallLayout& L) {
  size_t b = (size_t)L.nreal * sizeof(R) + (size_t)L.nint * sizeof(int);
  return (b + 15) & ~size_t(15);
}

template <typename R, int P>
__global__ void __launch_bounds__(P * 32) implsch_kernel(const DevTables<R> T, const ImplArgs<R> a) {
  extern __shared__ __align__(16) unsigned char smem[];
  R* sR = reinterpret_cast<R*>(smem);
  int* sI = reinterpret_cast<int*>(sR + T.lay.nreal);
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int i = tid; i < T.lay.nreal; i += nthr) sR[i] = T.small[i];
  for (int i = tid; i < T.lay.nint; i += nthr) sI[i] = T.ismall[i];
  const int NS = T.NS, KL = T.KL, LD = T.ld;
  const size_t wsb = warp_ws_bytes<R>(LD, T.ML, T.need_sp, T.scr);
  unsigned char* ws0 = smem + tables_bytes<R>(T.lay);
  const size_t foff = ws_f_offset<R>(LD, T.ML);  // F follows the interleaved {SL, FL} block
  const int ij0 = blockIdx.x * P;
  // stage the P spectra: consecutive threads take consecutive points of one bin
  for (int idx = tid; idx < P * NS; idx += nthr) {
    int p = idx % P, b = idx / P, ij = ij0 + p;
    int m = b / KL, k = b - m * KL;
    if (ij < a.nsea) reinterpret_cast<R*>(ws0 + p * wsb + foff)[k + LD * m] = a.fl3_in[ij + (size_t)a.ld * b];
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, ij = ij0 + warp;
  if (ij < a.nsea) {
    STabs<R> S;
    S.bind(sR, sI, T.lay);
    WarpWS<R> w;
    unsigned char* base = ws0 + warp * wsb;
    const int nrow = LD * T.ML;
    w.ld = LD; w.scr = T.scr;
    w.SF = reinterpret_cast<typename WarpWS<R>::R2*>(base);
    w.F = reinterpret_cast<R*>(base + foff);
    w.SP = T.need_sp ? w.F + nrow : nullptr;
    w.T = reinterpret_cast<R*>(base + ws_t_offset<R>(LD, T.ML, T.need_sp));
    w.LL = reinterpret_cast<uint8_t*>(w.T + 8 * T.scr);
    Src<R> src(T, S, w, lane, ij, a.indep[ij], a.u10[ij], a.udir[ij], a.roairn[ij], a.wstar[ij], a.depth[ij]);
    PointState<R> ps;
    ps.TAUW = a.tauw[ij];
    src.run(ps);
    if (lane == 0) {
      a.tauw[ij] = ps.TAUW; a.ustar[ij] = ps.USTAR; a.z0[ij] = ps.Z0;
      if (T.lcflx && a.fluxes)
        for (int q = 0; q < 7; ++q) a.fluxes[ij + (size_t)a.flx_ld * q] = ps.flx[q];
      if (!isfinite(ps.TAUW) || !isfinite(ps.USTAR) || !isfinite(ps.Z0)) atomicOr(a.status, 1);
    }
  }
  __syncthreads();
  for (int idx = tid; idx < P * NS; idx += nthr) {
    int p = idx % P, b = idx / P, ijs = ij0 + p;
    int m = b / KL, k = b - m * KL;
    if (ijs < a.nsea) {
      R v = reinterpret_cast<R*>(ws0 + p * wsb + foff)[k + LD * m];
      a.fl3[ijs + (size_t)a.ld * b] = v;
      if (!isfinite(v)) atomicOr(a.status, 1);
    }
  }
}

template <typename R> size_t implsch_smem_bytes(const DevTables<R>& T, int P) {
  return tables_bytes<R>(T.lay) + (size_t)P * warp_ws_bytes<R>(T.ld, T.ML, T.need_sp, T.scr);
}

// CTA shapes compiled: FP32 with 4, 6 or 8 sea points per CTA, FP64 with 2 or 4.
template <typename R, int P> cudaError_t set_smem_one(size_t bytes) {
  return cudaFuncSetAttribute(implsch_kernel<R, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}
template <typename R, int P> void launch_one(const DevTables<R>& T, const ImplArgs<R>& a, size_t smem, cudaStream_t s) {
  implsch_kernel<R, P><<<(a.nsea + P - 1) / P, P * 32, smem, s>>>(T, a);
}

template <typename R> cudaError_t implsch_set_max_smem(int P, size_t bytes) {
  if (sizeof(R) == 4) {
    if (P == 4) return set_smem_one<R, 4>(bytes);
    if (P == 6) return set_smem_one<R, 6>(bytes);
    if (P == 8) return set_smem_one<R, 8>(bytes);
  } else {
    if (P == 2) return set_smem_one<R, 2>(bytes);
    if (P == 4) return set_smem_one<R, 4>(bytes);
  }
  return cudaErrorInvalidValue;
}

template <typename R> cudaError_t launch_implsch(const DevTables<R>& T, const ImplArgs<R>& a, int P, cudaStream_t s) {
  if (a.nsea == 0) return cudaSuccess;
  size_t smem = implsch_smem_bytes(T, P);
  if (sizeof(R) == 4) {
    if (P == 4) launch_one<R, 4>(T, a, smem, s);
    else if (P == 6) launch_one<R, 6>(T, a, smem, s);
    else if (P == 8) launch_one<R, 8>(T, a, smem, s);
    else return cudaErrorInvalidValue;
  } else {
    if (P == 2) launch_one<R, 2>(T, a, smem, s);
    else if (P == 4) launch_one<R, 4>(T, a, smem, s);
    else return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template cudaError_t launch_implsch<float>(const DevTables<float>&, const ImplArgs<float>&, int, cudaStream_t);
template cudaError_t launch_implsch<double>(const DevTables<double>&, const ImplArgs<double>&, int, cudaStream_t);
template size_t implsch_smem_bytes<float>(const DevTables<float>&, int);
template size_t implsch_smem_bytes<double>(const DevTables<double>&, int);
template cudaError_t implsch_set_max_smem<float>(int, size_t);
template cudaError_t implsch_set_max_smem<double>(int, size_t);

}  // namespace wamgpu
