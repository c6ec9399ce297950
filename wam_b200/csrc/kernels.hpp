// Launchers shared between the translation units of libwamgpu.
#pragma once
#include <cuda_runtime.h>
#include <climits>
#include <cstring>
#include <algorithm>
#include "wamgpu_config.hpp"

namespace wamgpu {

template <typename R> struct PropArgs;

// CHECK_CFL coefficient classes, in the order the extrema kernel reports them
enum CflClass { CFL_LAT11 = 0, CFL_LAT21, CFL_LAT12, CFL_LAT22, CFL_LON1, CFL_LON2, CFL_TH1, CFL_TH2, CFL_SG1, CFL_SG2, CFL_SUM, CFL_NCLASS };

// Per-point inputs/outputs of one IMPLSCH launch (device pointers).
template <typename R> struct ImplArgs {
  int nsea, ld;
  const R* fl3_in;  // spectrum read (may equal fl3)
  R* fl3;           // spectrum written
  const R* u10; const R* udir; const R* roairn; const R* wstar; const R* depth; const int* indep;
  R* tauw; R* ustar; R* z0;
  R* fluxes;   // 7 x flx_ld or null
  int flx_ld;  // leading dimension of fluxes (the full NSEA when a launch covers a range of points)
  int* status; // bit 0: non-finite output
};

template <typename R> cudaError_t launch_implsch(const DevTables<R>& T, const ImplArgs<R>& a, int points_per_cta, cudaStream_t s);
template <typename R> size_t implsch_smem_bytes(const DevTables<R>& T, int points_per_cta);
template <typename R> cudaError_t implsch_set_max_smem(int points_per_cta, size_t bytes);

// PROPAGS over the frequency planes m0 .. m0+mcount-1 (mcount < 0: to ML).
template <typename R>
cudaError_t launch_propags(const PropArgs<R>& A, const R* f1, int ld1, R* f3, int ld3, cudaStream_t s, int m0 = 0,
                           int mcount = -1);
// True when a sub-step of plane m reads only plane m (no current refraction).
bool propags_planes_independent(int variant);
template <typename R> cudaError_t launch_cfl_extrema(const PropArgs<R>& A, long long* ext, int nsm, cudaStream_t s);
double cfl_decode(long long v, int precision);
cudaError_t static_scratch_address(void** p);

}  // namespace wamgpu
