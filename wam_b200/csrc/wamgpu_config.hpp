// Internal view of the C-ABI configuration plus the device-side table block.
#pragma once
#include "../../include/wamgpu.h"

namespace wamgpu {

using Config = wamgpu_config;

// Upper bounds of the spectral grid handled by the kernels (shared-memory
// sizing and per-lane register arrays).  wamgpu_create rejects larger grids.
constexpr int MAX_KL = 64;
constexpr int MAX_ML = 48;
constexpr int MAX_NK10 = 96;   // ST6 frequency axis extended to 10 Hz (LFACTOR)
constexpr int SCR = 96;        // per-warp per-frequency scratch length (>= MAX_ML, MAX_KL, MAX_NK10)

// The DIA coefficients RNLCOEF(1:25, MC) are stored RNL_STRIDE per MC,
// grouped for 4-wide loads: {0, 1, 2, 3}, {4, 13, 14, 15}, {16, -, -, -}
// (the tail factor and the weights of the eight gathers), then the target
// weights of each row kind: MM {20, 19, 23, 24}, MM1 {17, 18, 21, 22},
// MP {8, 7, 11, 12}, MP1 {5, 6, 9, 10} (0-based reference indices).  Each
// MC's block starts 16-byte aligned.  rnl_slot(i) is the slot of index i.
constexpr int RNL_STRIDE = 28;
__host__ __device__ constexpr int rnl_slot(int i) {
  constexpr int slot[25] = {0, 1, 2, 3, 4, 24, 25, 21, 20, 26, 27, 22, 23, 5, 6, 7, 8, 16, 17, 13, 12, 18, 19, 14, 15};
  return slot[i];
}

// Offsets (in elements) of the small tables inside the packed blocks that
// every IMPLSCH CTA stages into shared memory.
struct SmallLayout {
  // float block
  int FR, DF, DFIM, DFIMOFR, FR5, FRM5, RHOWG_DFIM, TH, COSTH, SINTH, DELFL, AF11, RNLCOEF, SATW, WTAUHF, SWELLFT,
      SIG10, DSII10;
  int nreal;
  // int block
  int K1W, K2W, K11W, K21W, INLCOEF, IKP, IKP1, IKM, IKM1, INDSAT;
  int nint;
};

// Everything the kernels need besides the per-point fields; passed by value.
template <typename R> struct DevTables {
  int KL, ML, NS, NDEPTH, MFRSTLW, MLSTHG, KFRH, NSDSNTH, NK10;
  int ld, scr, need_sp;  // shared-memory row stride (odd, >= KL), scratch row length, SPOS array kept
  int dia_batch;         // MCs per batch of the DIA's directions beyond the first 32 (KL > 32)
  unsigned long long dia_adj_starts[2];  // DIA^T: bit MC-1 set where a batch starts (MC <= 128; every later MC starts one)
  int iphys, shallow, isnonlin, lcflx;
  R DELTH, DELTR, INV_LOG_CO, MO_TAIL, MM1_TAIL, DELU, DAL1, DAL2, X0TAUHF;
  R BETAMAX, ZALP, ALPHA, TAUWSHELTER, CDFAC, DELT;
  SmallLayout lay;
  const R* small;      // packed float tables (global copy)
  const int* ismall;   // packed int tables (global copy)
  const R* TFAK;       // [(jd) + NDEPTH*m], jd 0-based
  const R* TCGOND;
  const R* FLMINFR;    // [(ju) + 300*m], ju 0-based
  const int4* diamc;   // per MC: 3 int4 of DIA row offsets, write flags and the AF11 index
  const int4* dslot;   // KL > 32: DIA batch slot entries, 4*(KL-32) for the forward, then as many for the adjoint
};

}  // namespace wamgpu
