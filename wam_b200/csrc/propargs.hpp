// Propagation variants and the per-point metadata block of the PROPAGS kernels
// (host and device view).
#pragma once
#include "wamgpu_config.hpp"

namespace wamgpu {

enum PropVariant : int {
  V_CART_DEEP = 0, V_CART_SHALLOW = 1, V_CART_DEEP_CUR = 2, V_CART_SHALLOW_CUR = 3,
  V_SPHER_DEEP = 4, V_SPHER_SHALLOW = 5, V_SPHER_DEEP_CURR = 6, V_SPHER_SHALLOW_CURR = 7
};

// Per-sea-point metadata (index i = 0-based local point; neighbour values are
// 1-based local numbers, 0 = land).  Arrays are of length n_ext (local points
// followed by halo points) unless noted.
template <typename R> struct PropArgs {
  int nsea, ld, KL, ML, variant, reduced, refr_d, spherical, counter, NDEPTH;
  int i0, i1;         // sea points the kernels update (0-based, [i0, i1)); the rest are halo points
  R DELPH0, DELTH0, DELTHR, DELFR0, rcounter;
  const int* klat;    // [i + nsea*(ic + 2*j)]   (nsea entries per slot)
  const int* klon;    // [i + nsea*dir]
  const R* wlat;      // [i + nsea*ic]
  const R* dpsn;      // [i + nsea*ic]
  const R* della0;    // [i]   (variant-specific longitude metric factor)
  const R* drgm;      // [i]   SINPH*DCO
  const int* indep;   // [n_ext] depth-table index (1-based), CGOND of point and neighbours
  const int* indep_g; // [i]   averaged depth index for refraction
  const R* ddphi;     // [i]   depth gradients (DDLAM already times DCO on spherical grids)
  const R* ddlam;
  const R* duphi; const R* dulam; const R* dvphi; const R* dvlam;  // current gradients
  const R* u; const R* v;    // [n_ext] currents (land slot reads as 0)
  const R* TCGOND; const R* TSIHKD; const R* TFAK;  // depth tables [(jd-1) + NDEPTH*m]
  const R* GOM; const R* FR;  // small tables (global)
  // SINTH/COSTH of this grid.  The struct is passed as a __grid_constant__
  // kernel parameter, so these are constant-bank reads (broadcast: every lane
  // of a warp reads the same direction), and every grid carries its own.
  R sinth[MAX_KL], costh[MAX_KL];
};

}  // namespace wamgpu
