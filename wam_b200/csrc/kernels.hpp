// Launchers shared between the translation units of libwamgpu.
#pragma once
#include <cuda_runtime.h>
#include <climits>
#include <cstring>
#include <algorithm>
#include "wamgpu_config.hpp"
#include "propargs.hpp"
#include "adjoint.cuh"

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
  const R* enh;  // MAKE_SHALLOW_SNL factors [ij + enh_ld*(mc-1)] when shallow && isnonlin != 0, else null
  int enh_ld;
  const R* wncg;  // ST6: WN then CG (ML values each) per point [ij * 2*ML], or null (formed in the step)
  int* status; // bit 0: non-finite output
  // test diagnostics of the integer decisions (null: off): diag[ij + diag_ld*q]
  // for q = JU, MIJ first, MIJ last, LFACTOR iterations; diag_ll[ij +
  // diag_ld*(b + NS*q)] the LLWS masks of the first and of the last SINPUT call
  int* diag = nullptr;
  uint8_t* diag_ll = nullptr;
  int diag_ld = 0;
  R* lfout = nullptr;  // ST6: per point the RTAU of LFACTOR's last round (0 without one), or null
};

template <typename R> cudaError_t launch_implsch(const DevTables<R>& T, const ImplArgs<R>& a, int points_per_cta, cudaStream_t s);
// WAVNU2's wavenumber and group velocity of every (sea point, frequency) from
// the depth, the same routine the ST6 step uses: out[ij * 2*ML + m] = WN,
// out[ij * 2*ML + ML + m] = CG.
template <typename R> cudaError_t launch_wavnu2(const DevTables<R>& T, const R* depth, int nsea, R* out, cudaStream_t s);
// Batched IMPLSCH over members that share their source tables T (one
// spectral grid and physics configuration): CTA b works for member g with
// first[g] <= b < first[g+1] (first[g] = sum of ceil(NSEA/P) over the members
// before g), whose per-point arguments are mem[g].
template <typename R>
cudaError_t launch_implsch_batch(const DevTables<R>& T, const ImplArgs<R>* mem, const int* first, int nmem, int nblocks,
                                 int points_per_cta, size_t smem, cudaStream_t s);
template <typename R> size_t implsch_smem_bytes(const DevTables<R>& T, int points_per_cta);
template <typename R> cudaError_t implsch_set_max_smem(int points_per_cta, size_t bytes);

// PROPAGS over the frequency planes m0 .. m0+mcount-1 (mcount < 0: to ML).
template <typename R>
cudaError_t launch_propags(const PropArgs<R>& A, const R* f1, int ld1, R* f3, int ld3, cudaStream_t s, int m0 = 0,
                           int mcount = -1);
// True when a sub-step of plane m reads only plane m (no current refraction).
bool propags_planes_independent(int variant);
// One member of a batched PROPAGS sub-step: its metadata, the buffers of
// this sub-step and the number of point blocks per frequency.
template <typename R> struct PropMember {
  PropArgs<R> A;
  const R* src;
  R* dst;
  int ld, nbi;
};
// All members of one coefficient family (variant, reduced grid, depth
// refraction taken from `family`) in one launch of bs-point CTAs (128 or 256);
// CTA b works for member g with first[g] <= b < first[g+1] (first[g] = sum of
// ML*nbi over the members before g).
template <typename R>
cudaError_t launch_propags_batch(const PropArgs<R>& family, const PropMember<R>* mem, const int* first, int nmem,
                                 int nblocks, int bs, cudaStream_t s);
template <typename R> cudaError_t launch_cfl_extrema(const PropArgs<R>& A, long long* ext, int nsm, cudaStream_t s);
double cfl_decode(long long v, int precision);
cudaError_t static_scratch_address(void** p);

// Arguments of the IMPLSCH tangent-linear and adjoint kernels (ST4, one sea
// point per thread).  work: deriv_work_bytes per point, masks: 2*KL*ML bytes
// per point, both laid out with the sea point fastest.
template <typename R> struct DerivArgs {
  adj::ATabs<R> A;
  int nsea, ld;
  const R *fl3_in, *tauw_in, *u10, *udir, *roairn, *wstar, *depth;
  const int* indep;
  const R* enh;
  int enh_ld;
  void* work;
  uint8_t* masks;
  // adjoint: in = adjoints of the outputs, out = adjoints of the inputs
  R *lam_fl3, *lam_tauw, *lam_u10;
  R* lam_out;  // where the adjoint kernel writes the input spectrum's adjoint (null: lam_fl3)
  const R* lfin;  // ST6: per point the RTAU of LFACTOR's last round of the forward step (null: iterate again)
  // tangent-linear
  const R *dfl3_in, *dtauw_in, *du10;
  R *fl3_out, *dfl3_out, *tauw_out, *dtauw_out, *ustar_out, *z0_out;
};
template <typename R> size_t deriv_work_bytes(int KL, int ML);

// Arguments of the integrated-output kernel (COMPUTE_OUTPUT_PARAMETER,
// wam_output_module.f90:481-640): one thread per sea point.  block receives
// parameter IP (the reference's numbering) at block[ij + block_ld*(IP-1)].
template <typename R> struct OutArgs {
  int nsea, ld, KL, ML, NDEPTH, shallow, from;
  const R* fl3;
  const R *u10, *udir, *tauw, *depth, *u, *v;  // u, v: currents or null
  R *ustar, *z0;                               // written by AIRSEA when USTAR is zero everywhere
  const int* indep;
  R* block;
  int block_ld;
  const R *FR, *DFIM, *DFIMOFR, *DFIM_FR, *DFIM_FR2, *MSSFD, *SINTH, *COSTH, *TFAK;
  const R *TH = nullptr, *C = nullptr;  // directions and deep-water phase speeds (swell separation)
  R MO_TAIL, MM1_TAIL, MP1_TAIL, MP2_TAIL;
  adj::ATabs<R> A;
  const unsigned long long* ustar_max;  // set by the launcher
};
// SWELL_SEPARATION without the partitioning: parameters 17-23 and 25-31 of
// a.block from the spectrum, UDIR and USTAR.
template <typename R> cudaError_t launch_swell(const OutArgs<R>& a, cudaStream_t s);
// PUT_ICE_SPEC / PUT_DRY_SPEC and PUT_ICE_PAR / PUT_DRY_PAR: data[(ij-1) +
// ld*row] = value for rows 0..nrows-1 and the 1-based sea points ij of the
// list that lie in lo..hi.
template <typename R>
cudaError_t launch_put_points(R* data, size_t ld, int nrows, const int* points, int n, int lo, int hi, R value,
                              cudaStream_t s);
// WAM_WIND: input wind components u_in, v_in [(i-1) + nx_in*(k-1)] to U10
// and UDIR of n sea points; tab holds I1, I2, K1, K2 (1-based, 4 blocks of
// n), w the weights DI, DK (2 blocks of n); equal != 0 copies point (I1, K1).
template <typename R>
cudaError_t launch_wind(const R* u_in, const R* v_in, int nx_in, int n, const int* tab, const R* w, int equal,
                        int code_in, R* us, R* ds, cudaStream_t s);
// Restart records (REAL, file order: position p holds point perm[p], 1-based,
// or p without perm) from rows b0..b0+nb-1 of a device array with the sea
// point fastest, and back.
template <typename R>
cudaError_t launch_restart_gather(const R* src, size_t ld, int nsea, const int* perm, int b0, int nb, float* out,
                                  cudaStream_t s);
template <typename R>
cudaError_t launch_restart_scatter(const float* in, int nsea, const int* perm, int b0, int nb, R* dst, size_t ld,
                                   cudaStream_t s);
// ustar_max: device word for MAXVAL(USTAR), or null to skip the AIRSEA check.
template <typename R> cudaError_t launch_output(const OutArgs<R>& a, unsigned long long* ustar_max, cudaStream_t s);
template <typename R> cudaError_t launch_implsch_adj(const DevTables<R>& T, const DerivArgs<R>& a, cudaStream_t s);
template <typename R> cudaError_t launch_implsch_tl(const DerivArgs<R>& a, cudaStream_t s);
// Transpose of one PROPAGS sub-step: lam_old (zeroed by the caller) +=
// P^T lam_new, by atomic adds into the neighbours' bins.
template <typename R>
cudaError_t launch_propags_adj(const PropArgs<R>& A, const R* lam_new, int ld1, R* lam_old, int ld3, cudaStream_t s);

}  // namespace wamgpu
