// IMPLSCH kernel entry: CTA of P warps = P consecutive sea points.
#include "implsch.cuh"
#include "kernels.hpp"
#include <mutex>

namespace wamgpu {

// One CTA: sea points blk*P .. blk*P+P-1 of the launch's arguments.
template <typename R, int P>
__device__ __forceinline__ void implsch_cta(const DevTables<R>& T, const ImplArgs<R>& a, int blk, unsigned char* smem) {
  R* sR = reinterpret_cast<R*>(smem);
  int* sI = reinterpret_cast<int*>(sR + T.lay.nreal);
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int NS = T.NS, KL = T.KL, LD = T.ld;
  const size_t wsb = warp_ws_bytes<R>(LD, T.ML, T.need_sp, T.scr);
  unsigned char* ws0 = smem + tables_bytes<R>(T.lay);
  const size_t foff = ws_f_offset<R>(LD, T.ML);  // F follows the interleaved {SL, FL} block
  const int ij0 = blk * P;
  // stage the P spectra: consecutive threads take consecutive points of one
  // bin.  With 32*P threads, thread t always takes point t mod P and the bins
  // t div P + 32 j, whose (m, k) advance by a carry instead of a division.
  const int tp = tid % P, tb = tid / P, dq = 32 / KL, dr = 32 - dq * KL;
  {
    const int ij = min(ij0 + tp, a.nsea - 1);
    R* dstF = reinterpret_cast<R*>(ws0 + tp * wsb + foff);
    const R* src = a.fl3_in + ij;
    int m = tb / KL, k = tb - m * KL;
    for (int b = tb; b < NS; b += 32) {
      const unsigned sa = (unsigned)__cvta_generic_to_shared(dstF + k + LD * m);
      const R* g = src + (size_t)a.ld * b;
      if (sizeof(R) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(g) : "memory");
      else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
      k += dr; m += dq;
      if (k >= KL) { k -= KL; ++m; }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int i = tid; i < T.lay.nreal; i += nthr) sR[i] = T.small[i];
  for (int i = tid; i < T.lay.nint; i += nthr) sI[i] = T.ismall[i];
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  // every warp runs the step (its phases end in CTA barriers); a warp past the
  // last sea point repeats the last point and writes nothing
  const int warp = tid >> 5, lane = tid & 31, ij = min(ij0 + warp, a.nsea - 1);
  const bool real = ij0 + warp < a.nsea;
  {
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
    Src<R> src(T, S, w, lane, ij, a.indep[ij], a.u10[ij], a.udir[ij], a.roairn[ij], a.wstar[ij], a.depth[ij], a.enh,
               a.enh_ld);
    src.wncg = a.wncg ? a.wncg + (size_t)ij * 2 * T.ML : nullptr;
    if (a.diag_ll && real) { src.dll = a.diag_ll + ij; src.dll_ld = (size_t)a.diag_ld; }
    if (a.lfout && real) src.lfout = a.lfout + ij;
    PointState<R> ps;
    ps.TAUW = a.tauw[ij];
    src.run(ps);
    if (lane == 0 && real) {
      a.tauw[ij] = ps.TAUW; a.ustar[ij] = ps.USTAR; a.z0[ij] = ps.Z0;
      if (a.diag) {
        a.diag[ij] = ps.JU; a.diag[ij + (size_t)a.diag_ld] = ps.MIJ1;
        a.diag[ij + 2 * (size_t)a.diag_ld] = ps.MIJ2; a.diag[ij + 3 * (size_t)a.diag_ld] = ps.LFIT;
      }
      if (T.lcflx && a.fluxes)
        for (int q = 0; q < 7; ++q) a.fluxes[ij + (size_t)a.flx_ld * q] = ps.flx[q];
      if (!isfinite(ps.TAUW) || !isfinite(ps.USTAR) || !isfinite(ps.Z0)) atomicOr(a.status, 1);
    }
  }
  __syncthreads();
  if (ij0 + tp < a.nsea) {
    const R* srcF = reinterpret_cast<const R*>(ws0 + tp * wsb + foff);
    R* dst = a.fl3 + ij0 + tp;
    bool finite = true;
    int m = tb / KL, k = tb - m * KL;
    for (int b = tb; b < NS; b += 32) {
      const R v = srcF[k + LD * m];
      dst[(size_t)a.ld * b] = v;
      finite = finite && isfinite(v);
      k += dr; m += dq;
      if (k >= KL) { k -= KL; ++m; }
    }
    if (!finite) atomicOr(a.status, 1);
  }
}

template <typename R, int P>
__global__ void __launch_bounds__(P * 32) implsch_kernel(const __grid_constant__ DevTables<R> T, const ImplArgs<R> a) {
  extern __shared__ __align__(16) unsigned char smem[];
  implsch_cta<R, P>(T, a, blockIdx.x, smem);
}

// Batched form: the CTAs of all members that share the source tables T (one
// spectral grid and physics configuration) in one launch.  CTA b belongs to
// member g with first[g] <= b < first[g + 1]; the member's per-point argument
// block is copied into shared memory first, T stays a kernel parameter.
template <typename R, int P>
__global__ void __launch_bounds__(P * 32) implsch_batch_kernel(const __grid_constant__ DevTables<R> T,
                                                              const ImplArgs<R>* __restrict__ mem,
                                                              const int* __restrict__ first, int nmem) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(16) ImplArgs<R> sa;
  __shared__ int sg;
  if (threadIdx.x == 0) {
    int lo = 0, hi = nmem - 1;  // last g with first[g] <= blockIdx.x
    while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (first[mid] <= (int)blockIdx.x) lo = mid; else hi = mid - 1; }
    sg = lo;
  }
  __syncthreads();
  const int g = sg;
  {
    const int nw = (int)(sizeof(ImplArgs<R>) / sizeof(int));
    const int* src = reinterpret_cast<const int*>(mem + g);
    int* dst = reinterpret_cast<int*>(&sa);
    for (int q = threadIdx.x; q < nw; q += blockDim.x) dst[q] = src[q];
  }
  __syncthreads();
  implsch_cta<R, P>(T, sa, (int)blockIdx.x - first[g], smem);
}

template <typename R>
__global__ void __launch_bounds__(256) wavnu2_kernel(const __grid_constant__ DevTables<R> T, const R* __restrict__ depth,
                                                     int nsea, R* __restrict__ out) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int ML = T.ML;
  if (t >= (size_t)nsea * ML) return;
  const int ij = (int)(t / ML), m = (int)(t - (size_t)ij * ML);
  const R w0 = dabs(Phys<R>::ZPI * T.small[T.lay.FR + m]);
  wavnu2_one(w0, depth[ij], out[(size_t)ij * 2 * ML + m], out[(size_t)ij * 2 * ML + ML + m]);
}

template <typename R> cudaError_t launch_wavnu2(const DevTables<R>& T, const R* depth, int nsea, R* out, cudaStream_t s) {
  const size_t n = (size_t)nsea * T.ML;
  if (n == 0) return cudaSuccess;
  wavnu2_kernel<R><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(T, depth, nsea, out);
  return cudaGetLastError();
}
template cudaError_t launch_wavnu2<float>(const DevTables<float>&, const float*, int, float*, cudaStream_t);
template cudaError_t launch_wavnu2<double>(const DevTables<double>&, const double*, int, double*, cudaStream_t);

template <typename R> size_t implsch_smem_bytes(const DevTables<R>& T, int P) {
  return tables_bytes<R>(T.lay) + (size_t)P * warp_ws_bytes<R>(T.ld, T.ML, T.need_sp, T.scr);
}

// CTA shapes compiled: FP32 with 4, 6 or 8 sea points per CTA, FP64 with 2 or 4.
template <typename R, int P> cudaError_t set_smem_one(size_t bytes) {
  cudaError_t e = cudaFuncSetAttribute(implsch_kernel<R, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(implsch_batch_kernel<R, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}
template <typename R, int P>
void launch_batch_one(const DevTables<R>& T, const ImplArgs<R>* mem, const int* first, int nmem, int nblocks, size_t smem,
                      cudaStream_t s) {
  implsch_batch_kernel<R, P><<<nblocks, P * 32, smem, s>>>(T, mem, first, nmem);
}
template <typename R, int P> void launch_one(const DevTables<R>& T, const ImplArgs<R>& a, size_t smem, cudaStream_t s) {
  implsch_kernel<R, P><<<(a.nsea + P - 1) / P, P * 32, smem, s>>>(T, a);
}

// The opt-in shared-memory limit of a kernel instance is process state of
// the device: it is only ever raised, so a batch or a context with a small
// spectrum never lowers it under another live context's need.
template <typename R> cudaError_t implsch_set_max_smem(int P, size_t bytes) {
  static std::mutex mu;
  static size_t cur[2][64][9] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || P < 0 || P > 8) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(mu);
  size_t& c = cur[sizeof(R) == 4 ? 0 : 1][dev][P];
  if (bytes <= c) return cudaSuccess;
  if (sizeof(R) == 4) {
    if (P == 4) e = set_smem_one<R, 4>(bytes);
    else if (P == 6) e = set_smem_one<R, 6>(bytes);
    else if (P == 8) e = set_smem_one<R, 8>(bytes);
    else return cudaErrorInvalidValue;
  } else {
    if (P == 2) e = set_smem_one<R, 2>(bytes);
    else if (P == 4) e = set_smem_one<R, 4>(bytes);
    else return cudaErrorInvalidValue;
  }
  if (e == cudaSuccess) c = bytes;
  return e;
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

template <typename R>
cudaError_t launch_implsch_batch(const DevTables<R>& T, const ImplArgs<R>* mem, const int* first, int nmem, int nblocks,
                                 int P, size_t smem, cudaStream_t s) {
  if (nblocks == 0) return cudaSuccess;
  if (sizeof(R) == 4) {
    if (P == 4) launch_batch_one<R, 4>(T, mem, first, nmem, nblocks, smem, s);
    else if (P == 6) launch_batch_one<R, 6>(T, mem, first, nmem, nblocks, smem, s);
    else if (P == 8) launch_batch_one<R, 8>(T, mem, first, nmem, nblocks, smem, s);
    else return cudaErrorInvalidValue;
  } else {
    if (P == 2) launch_batch_one<R, 2>(T, mem, first, nmem, nblocks, smem, s);
    else if (P == 4) launch_batch_one<R, 4>(T, mem, first, nmem, nblocks, smem, s);
    else return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template cudaError_t launch_implsch_batch<float>(const DevTables<float>&, const ImplArgs<float>*, const int*, int, int, int,
                                                 size_t, cudaStream_t);
template cudaError_t launch_implsch_batch<double>(const DevTables<double>&, const ImplArgs<double>*, const int*, int, int,
                                                  int, size_t, cudaStream_t);
template cudaError_t launch_implsch<float>(const DevTables<float>&, const ImplArgs<float>&, int, cudaStream_t);
template cudaError_t launch_implsch<double>(const DevTables<double>&, const ImplArgs<double>&, int, cudaStream_t);
template size_t implsch_smem_bytes<float>(const DevTables<float>&, int);
template size_t implsch_smem_bytes<double>(const DevTables<double>&, int);
template cudaError_t implsch_set_max_smem<float>(int, size_t);
template cudaError_t implsch_set_max_smem<double>(int, size_t);

}  // namespace wamgpu
