/*
 * wamgpu.h - C ABI of the B200 (sm_100a) implementation of WAM Cycle 7's
 * per-time-step hot path: the implicit source-term integration IMPLSCH
 * (ST4 / IPHYS=1 and ST6 / IPHYS=2, with the DIA nonlinear transfer) and the
 * spectral propagation PROPAGS with depth and current refraction.
 *
 * The Fortran driver binds these entry points through ISO_C_BINDING behind
 * the reference's own module procedure names.  Every
 * entry point that replaces a reference procedure cites it; references are
 * myWAveModel/WAM file:line.
 *
 * Conventions
 *  - Spectra use the reference layout FL3(IJ,K,M): sea point fastest, then
 *    direction K (1..KL), then frequency M (1..ML), single precision.
 *  - Index tables keep the reference convention: 1-based sea point numbers,
 *    0 for a land neighbour (KLAT, KLON), 1-based depth-table index (INDEP).
 *  - Every call returns 0 on success and a negative WAMGPU_E* code on
 *    failure; wamgpu_last_error() then holds a message.  There is no CPU
 *    fallback: without a usable CUDA device every call fails.
 *  - One context per rank/thread; work is ordered on the context's CUDA
 *    stream.  *_host calls are synchronous; *_dev calls are asynchronous on the
 *    stream passed (NULL = the context stream).
 */
#ifndef WAMGPU_H
#define WAMGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define WAMGPU_API __attribute__((visibility("default")))
#else
#define WAMGPU_API
#endif

#define WAMGPU_OK 0
#define WAMGPU_E_ARG -1       /* invalid argument or unsupported option      */
#define WAMGPU_E_CUDA -2      /* CUDA runtime error                           */
#define WAMGPU_E_STATE -3     /* call out of order (e.g. no grid yet)         */
#define WAMGPU_E_CFL -4       /* negative propagation coefficient (CHECK_CFL) */
#define WAMGPU_E_NOMEM -5     /* device allocation failed                     */
#define WAMGPU_E_NUMERIC -6   /* non-finite values detected in outputs        */
#define WAMGPU_E_TIMEOUT -7   /* reserved: a bounded device wait expired; no  */
                              /* entry point returns it yet                   */

typedef struct wamgpu_ctx wamgpu_ctx;

/* Model configuration.  Field meaning follows the reference module variables
 * after INITMDL (initmdl.f90:137-212): effective BETAMAX, ZALP, ALPHA and
 * TAUWSHELTER after the ST4 swap and the ML<=30 ALPHA rule (initmdl.f90:153-160).
 * Layout is shared with the Fortran shim (BIND(C) derived type). */
typedef struct wamgpu_config {
  int kl, ml;                 /* KL directions, ML frequencies (wam_fre_dir_module.f90:38-39) */
  double fr1; int iref;       /* SET_FRE_DIR(N_DIR,N_FRE,FR1,IREF), fre_dir:122 */
  int iphys;                  /* 1 = ST4 (Ardhuin), 2 = ST6 */
  int shallow_run, spherical_run, refraction_d_run, refraction_c_run, reduced_grid;
  int isnonlin, lcflx;        /* SNL depth scaling option; compute surface fluxes */
  int idelt, idelpro;         /* source and propagation time steps [s] */
  double betamax, zalp, alpha, tauwshelter, cdfac;
  int ndepth; double deptha, depthd;  /* shallow-water table (wam_tables_module.f90:76-79) */
  double delphi;              /* latitude increment [m] (wam_grid_module DELPHI) */
  int precision;              /* 4 = FP32 (production), 8 = FP64 reference run of the same kernels */
  int device;                 /* CUDA device ordinal */
} wamgpu_config;

/* Creates a context and builds the static spectral tables on the host:
 * MAKE_FRE_DIR (wam_fre_dir_module.f90:297-459), MAKE_SHALLOW_TABLES
 * (wam_tables_module.f90:388-464), MIN_ENERGY (:315-384), NLWEIGT and
 * INIT_SNONLIN (wam_source_module.f90:1056-1523), TABU_SWELLFT (:3360),
 * INIT_SDISSP_ARD (:3419), INIT_X0TAUHF (:3784); then uploads them.
 * Replaces the table part of PREPARE_SOURCE (wam_source_module.f90:704). */
WAMGPU_API int wamgpu_create(const wamgpu_config* cfg, wamgpu_ctx** out);
WAMGPU_API int wamgpu_destroy(wamgpu_ctx* ctx);
WAMGPU_API const char* wamgpu_last_error(const wamgpu_ctx* ctx);
WAMGPU_API int wamgpu_config_size(void);

/* Reference-convention copy of a host table (names as in the reference,
 * e.g. "FR", "TFAK", "IKP", "K1W", "INDICESSAT"); returns the element count
 * when out is NULL.  Float tables go to fout, integer tables to iout. */
WAMGPU_API int wamgpu_get_table(const wamgpu_ctx* ctx, const char* name, float* fout, int* iout);

/* The same tables computed on the host without a context or a GPU (for a
 * driver that checks its own PREPARE_SOURCE tables against the library's). */
WAMGPU_API int wamgpu_host_table(const wamgpu_config* cfg, const char* name, float* fout, int* iout);

/* Grid module arrays for this rank's NSEA sea points (wam_grid_module.f90:
 * KLAT(NSEA,2,2), KLON(NSEA,2), WLAT(NSEA,2), KFROMIJ(NSEA)) and the
 * per-latitude SINPH, COSPH, DELLAM of the NY rows; computes DCO and DPSN
 * (wam_initial_module.f90:204-214). */
WAMGPU_API int wamgpu_set_grid(wamgpu_ctx* ctx, int nsea, const int* klat, const int* klon, const float* wlat,
                    const int* kfromij, int ny, const float* sinph, const float* cosph, const float* dellam);

/* Sea-point water depth [m] (WAM_MODEL_MODULE DEPTH) and currents U, V
 * [m/s] (NULL = zero).  Take effect at the next wamgpu_prepare_propagation. */
WAMGPU_API int wamgpu_set_depth(wamgpu_ctx* ctx, const float* depth);
WAMGPU_API int wamgpu_set_current(wamgpu_ctx* ctx, const float* u, const float* v);

/* PREPARE_PROPAGATION (wam_propagation_module.f90:279-598): INDEP, CGOND,
 * depth/current gradients, refraction terms, the propagation coefficients
 * and CHECK_CFL (:1917-2138) with COUNTER sub-stepping.  Returns
 * WAMGPU_E_CFL where the reference calls ABORT1 (negative coefficient). */
WAMGPU_API int wamgpu_prepare_propagation(wamgpu_ctx* ctx, float* total_cfl, int* counter);

/* MAKE_SHALLOW_SNL (wam_source_module.f90:975-1048) for ISNONLIN != 0 and the
 * remaining per-point source preparation; call after set_depth. */
WAMGPU_API int wamgpu_prepare_source(wamgpu_ctx* ctx);

/* INDEP(NSEA) as computed by prepare_propagation (propagation:327-332). */
WAMGPU_API int wamgpu_get_indep(const wamgpu_ctx* ctx, int* indep);

/* IMPLSCH(FL3, U10, UDIR, TAUW, USTAR, Z0, ROAIRN, WSTAR, DEPTH, INDEP)
 * (wam_source_module.f90:374-700) on host buffers: copies in, integrates one
 * source step of IDELT seconds on the device, copies FL3, TAUW, USTAR, Z0
 * back.  nsea must equal the grid's NSEA; depth/indep may be NULL to use the
 * context's own.  When LCFLX is set the flux-module arrays (wam_flux_module
 * PHIOC, TAUOC_X, TAUOC_Y, PHIBOT, TAUBOT_X, TAUBOT_Y, PHIAW) are kept on the
 * device; read them with wamgpu_get_fluxes. */
WAMGPU_API int wamgpu_implsch_host(wamgpu_ctx* ctx, float* fl3, const float* u10, const float* udir, float* tauw, float* ustar,
                        float* z0, const float* roairn, const float* wstar, const float* depth, const int* indep);

/* PROPAGS(F3) (wam_propagation_module.f90:635-829) on a host buffer: COUNTER
 * upwind sub-steps of IDELPRO/COUNTER seconds each. */
WAMGPU_API int wamgpu_propags_host(wamgpu_ctx* ctx, float* f3);

/* Device-pointer forms for callers that keep the model state resident on the
 * GPU.  fl3 has leading dimension ld >= NSEA (elements); pointer element type
 * is float for precision 4 and double for precision 8.  stream is a
 * cudaStream_t (NULL = context stream).  wamgpu_propags_dev takes an
 * optional scratch spectrum of the same shape (NULL = context-owned). */
WAMGPU_API int wamgpu_implsch_dev(wamgpu_ctx* ctx, void* fl3, int ld, const void* u10, const void* udir, void* tauw, void* ustar,
                       void* z0, const void* roairn, const void* wstar, void* stream);
WAMGPU_API int wamgpu_propags_dev(wamgpu_ctx* ctx, void* f3, int ld, void* scratch, void* stream);

/* Fixed-scratch form of wamgpu_propags_dev.  NO COUNTERPART IN THE REFERENCE
 * (its PROPAGS, wam_propagation_module.f90:635-829, sub-steps through a
 * local array of the model).  It serves callers that can neither hand in a
 * scratch spectrum nor let the library cudaMalloc one: hosts whose free
 * device memory is held by another allocator (the allocation would fail)
 * and pipelines that must not pass through the device-wide synchronisation
 * of the cudaFree that replacing a grown buffer implies.
 *  - The F1 ping-pong buffer of the COUNTER sub-steps is one file-scope
 *    device array of WAMGPU_STATIC_SCRATCH_BYTES per device.  A spectrum of
 *    more than that (ld*KL*ML*element size) is rejected with WAMGPU_E_ARG
 *    before any work is queued.
 *  - The first call on a device looks the array's address up
 *    (cudaGetSymbolAddress, which may load the module) and keeps it for the
 *    process; make that first call before any stream capture.
 *  - Nothing is allocated, freed or cleared: every scratch element a call
 *    reads it wrote earlier in the same call.  This holds for the whole
 *    grid only, so a context with an owned range (wamgpu_set_owned) is
 *    rejected with WAMGPU_E_ARG; a band driver sub-steps with
 *    wamgpu_propags_substep_dev instead.
 *  - The looked-up address belongs to the device's primary context: do not
 *    use the library across a cudaDeviceReset (which invalidates every
 *    context and buffer of the library as well).
 *  - There is ONE array per device: calls whose GPU work overlaps (other
 *    streams, other contexts on the same device) race on it; order them on
 *    one stream.
 *  - Kernel timing (wamgpu_set_timing) does not cover this entry point. */
#define WAMGPU_STATIC_SCRATCH_BYTES 33554432
WAMGPU_API int wamgpu_propags_dev_static(wamgpu_ctx* ctx, void* f3, int ld, void* stream);

/* One pass of the WAMODEL PROP/PHYSICS loop body (wamodel.f90:286-360):
 * nprop PROPAGS calls (IDELT/IDELPRO of them per source step) followed by
 * one IMPLSCH, with the spectrum resident on the device for the whole pass.
 * The _host form copies FL3 and the per-point fields in once and back once
 * (FP32 contexts), in chunks of consecutive sea points: a chunk goes up on
 * one copy stream, is propagated as soon as it and its neighbour chunks have
 * arrived (the sub-steps of the chunks run as a wavefront), is integrated,
 * and comes down on a second copy stream, so that both copy directions and
 * the kernels overlap.  Host buffers should be pinned for the copies to
 * overlap.  The _dev form works on caller-owned device buffers. */
WAMGPU_API int wamgpu_step_dev(wamgpu_ctx* ctx, void* fl3, int ld, void* scratch, int nprop, const void* u10,
                               const void* udir, void* tauw, void* ustar, void* z0, const void* roairn,
                               const void* wstar, void* stream);
WAMGPU_API int wamgpu_step_host(wamgpu_ctx* ctx, float* fl3, int nprop, const float* u10, const float* udir,
                                float* tauw, float* ustar, float* z0, const float* roairn, const float* wstar);

/* Flux-module arrays of the last LCFLX step, 7 blocks of NSEA in the order
 * PHIOC, TAUOC_X, TAUOC_Y, PHIBOT, TAUBOT_X, TAUBOT_Y, PHIAW (host copy). */
WAMGPU_API int wamgpu_get_fluxes(wamgpu_ctx* ctx, float* out7);

/* Kernel timing (tracing): while enabled, every PROPAGS and IMPLSCH launch is
 * bracketed by CUDA events on its stream.  wamgpu_get_timing waits for them
 * and returns the summed milliseconds and launch counts since the last call:
 * ms[0]/count[0] for PROPAGS, ms[1]/count[1] for IMPLSCH. */
WAMGPU_API int wamgpu_set_timing(wamgpu_ctx* ctx, int enable);
WAMGPU_API int wamgpu_get_timing(wamgpu_ctx* ctx, float* ms, int* count);

/* One grid over several ranks, in latitude bands as in the reference's MPI
 * decomposition: each rank owns a contiguous range NIJS..NIJL of the
 * south-to-north ordered sea points and reads its neighbours' spectra from a
 * halo (wam_mpi_comp_module.f90:1063-1095).  The reference packs exactly the
 * needed neighbour points into NINF..NSUP; here a rank's context holds the
 * contiguous index range that contains them (owned points plus halo,
 * neighbour numbers local to it), which costs a few more exchanged points and
 * gives the same results.
 *  - wamgpu_set_owned (before wamgpu_prepare_propagation) makes the kernels
 *    update only sea points i0..i1-1 (0-based).  CHECK_CFL then covers the
 *    owned points, IMPLSCH integrates them, and PROPAGS writes them and
 *    reads the halo points as the caller left them.
 *  - wamgpu_set_counter installs the COUNTER agreed over all ranks: the
 *    largest of the ranks' own values, which is CEILING of the global CFL
 *    maximum as CHECK_CFL computes it over all processors
 *    (propagation:2021-2130).
 *  - wamgpu_propags_substep_dev runs one sub-step of IDELPRO/COUNTER seconds
 *    from src to dst.  A band driver refreshes the halo of src before every
 *    sub-step, as PROPAGS exchanges it before each one (propagation:
 *    704-709).  The multi-sub-step entry points above do not exchange. */
WAMGPU_API int wamgpu_set_owned(wamgpu_ctx* ctx, int i0, int i1);
WAMGPU_API int wamgpu_set_counter(wamgpu_ctx* ctx, int counter);
WAMGPU_API int wamgpu_propags_substep_dev(wamgpu_ctx* ctx, const void* src, void* dst, int ld, void* stream);
/* The same sub-step over the sea points i0..i1-1 only (0-based, inside the
 * owned range).  A point further than the halo width from both ends of the
 * owned range reads no halo point, so a band driver sub-steps those interior
 * points while its halo exchange (mpi_exchng, wam_mpi_comp_module.f90:
 * 1466-1626) is in flight and the points near the band edges after it.
 * wamgpu_get_halo_width returns that width: the largest |neighbour - point|
 * over KLAT/KLON, in sea points (or a negative code without a grid). */
WAMGPU_API int wamgpu_propags_substep_range_dev(wamgpu_ctx* ctx, const void* src, void* dst, int ld, int i0, int i1,
                                                void* stream);
WAMGPU_API int wamgpu_get_halo_width(const wamgpu_ctx* ctx);

/* Batched ensembles.  No single counterpart in the reference, where each
 * member is a separate WAMODEL run calling PROPAGS (propagation:635-829) and
 * IMPLSCH (source:374-700).  A batch advances many prepared member contexts
 * of one precision on one device, each with its own grid size, KL/ML and
 * physics: one pass runs every member's IDELT/IDELPRO x COUNTER PROPAGS
 * sub-steps and then its IMPLSCH, with one launch per sub-step and
 * coefficient family and one IMPLSCH launch for all members.  Results are
 * bit-identical to wamgpu_step_dev of each member.
 *  - wamgpu_batch_set_member gives member g's device state, as for
 *    wamgpu_step_dev (scratch is required).
 *  - IMPLSCH runs one launch per class of members that share their source
 *    tables (spectral grid and physics configuration), so each launch keeps
 *    the occupancy of its own workspace size.
 *  - wamgpu_batch_tune times the compiled CTA shapes on the members' state,
 *    writing only scratch: points per PROPAGS CTA, and sea points per IMPLSCH
 *    CTA for each class.  It keeps the fastest and returns the PROPAGS value
 *    and the IMPLSCH value of the class with the most sea points.
 *  - wamgpu_batch_step runs one pass on `stream` (NULL = the first member's
 *    stream); after wamgpu_batch_capture it replays the captured CUDA graph.
 *    wamgpu_batch_capture records one pass as a CUDA graph; setting a
 *    member's state again discards it.
 *  - wamgpu_batch_sync waits for the stream and checks every member's
 *    non-finite flag. */
typedef struct wamgpu_batch wamgpu_batch;
WAMGPU_API int wamgpu_batch_create(wamgpu_ctx* const* members, int n, wamgpu_batch** out);
WAMGPU_API int wamgpu_batch_destroy(wamgpu_batch* b);
WAMGPU_API const char* wamgpu_batch_last_error(const wamgpu_batch* b);
WAMGPU_API int wamgpu_batch_set_member(wamgpu_batch* b, int g, void* fl3, int ld, void* scratch, const void* u10,
                                       const void* udir, void* tauw, void* ustar, void* z0, const void* roairn,
                                       const void* wstar);
WAMGPU_API int wamgpu_batch_tune(wamgpu_batch* b, void* stream, int* points_per_cta, int* propags_block);
WAMGPU_API int wamgpu_batch_step(wamgpu_batch* b, void* stream);
WAMGPU_API int wamgpu_batch_capture(wamgpu_batch* b, void* stream);
WAMGPU_API int wamgpu_batch_sync(wamgpu_batch* b);

/* Derivatives of one WAMODEL pass.  The reference has no tangent-linear or
 * adjoint code; these differentiate its forward procedures as they stand, and
 * are checked against central finite differences of the forward path and
 * against each other (<TL dx, ly> = <dx, ADJ ly>).
 *  - wamgpu_implsch_tl_dev: IMPLSCH (source:374-700) for ST4 (IPHYS=1) and
 *    its tangent-linear in one pass.  Inputs FL3 (fl3_in), TAUW and U10 with
 *    their perturbations dfl3_in, dtauw_in, du10; outputs the new spectrum
 *    and TAUW with their perturbations.  UDIR, ROAIRN, WSTAR and the depth
 *    are held fixed.  The branch decisions of the forward pass (MAX/MIN
 *    selections, the high-frequency tail mask, the limiter) are frozen at
 *    the base state, as a tangent-linear model takes them.
 *  - wamgpu_implsch_adj_dev: the adjoint of the same map.  It recomputes the
 *    forward pass from its inputs (the checkpoint: FL3, TAUW, U10 before
 *    IMPLSCH) and maps lam_fl3 (in: adjoint of the new FL3, out: adjoint of
 *    the old one), lam_tauw (in/out likewise) and lam_u10 (out, overwritten)
 *    in place.
 *  - wamgpu_propags_adj_dev: the transpose of PROPAGS (propagation:635-829),
 *    which is linear in FL3: the COUNTER sub-steps in reverse order, each a
 *    scatter of lam back to the points and bins it was gathered from.
 *    scratch (ld x KL x ML values, NULL = a context-owned buffer) holds the
 *    alternate sub-step; lam_f3 is updated in place.
 * All three cover the whole grid of a context (no owned range), need
 * wamgpu_prepare_propagation (and wamgpu_prepare_source with ISNONLIN != 0
 * in shallow water), and work in the context's precision. */
WAMGPU_API int wamgpu_implsch_tl_dev(wamgpu_ctx* ctx, const void* fl3_in, const void* dfl3_in, int ld,
                                     const void* tauw_in, const void* dtauw_in, const void* u10, const void* du10,
                                     const void* udir, const void* roairn, const void* wstar, void* fl3_out,
                                     void* dfl3_out, void* tauw_out, void* dtauw_out, void* stream);
WAMGPU_API int wamgpu_implsch_adj_dev(wamgpu_ctx* ctx, const void* fl3_in, int ld, const void* tauw_in,
                                      const void* u10, const void* udir, const void* roairn, const void* wstar,
                                      void* lam_fl3, void* lam_tauw, void* lam_u10, void* stream);
WAMGPU_API int wamgpu_propags_adj_dev(wamgpu_ctx* ctx, void* lam_f3, int ld, void* scratch, void* stream);

/* Checkpointed assimilation windows, built on the derivative entry points
 * (no reference counterpart).  A window of source steps runs forward with
 * wamgpu_step_ckpt_dev, one checkpoint slot per step, and backward with
 * wamgpu_step_adj_dev over the slots in reverse order; the driver adds its
 * observation terms to lam_fl3 between steps.
 *  - wamgpu_checkpoint_reserve keeps room on the device for n checkpoints of
 *    spectra with leading dimension ld (n = 0 releases it).  A checkpoint is
 *    the spectrum entering IMPLSCH, TAUW and U10 before it, and for ST6 the
 *    RTAU of LFACTOR's last round (the adjoint repeats that round only):
 *    ld*KL*ML + 3*NSEA values.
 *  - wamgpu_step_ckpt_dev is wamgpu_step_dev (WAMODEL's PROP/PHYSICS pass,
 *    wamodel.f90:286-360) that also stores checkpoint `slot`.
 *  - wamgpu_step_adj_dev is the adjoint of that step: wamgpu_implsch_adj_dev
 *    at the checkpoint, then nprop x wamgpu_propags_adj_dev.  lam_fl3 and
 *    lam_tauw map in place from the step's output to its input; lam_u10
 *    receives the adjoint of the step's U10.  scratch as for
 *    wamgpu_propags_adj_dev.
 * ld must be the one given to wamgpu_checkpoint_reserve. */
WAMGPU_API int wamgpu_checkpoint_reserve(wamgpu_ctx* ctx, int n, int ld);
WAMGPU_API int wamgpu_step_ckpt_dev(wamgpu_ctx* ctx, int slot, void* fl3, int ld, void* scratch, int nprop,
                                    const void* u10, const void* udir, void* tauw, void* ustar, void* z0,
                                    const void* roairn, const void* wstar, void* stream);
WAMGPU_API int wamgpu_step_adj_dev(wamgpu_ctx* ctx, int slot, int nprop, void* lam_fl3, int ld, void* lam_tauw,
                                   void* lam_u10, const void* udir, const void* roairn, const void* wstar,
                                   void* scratch, void* stream);

/* Test diagnostics of IMPLSCH's integer decisions.  No counterpart in the
 * reference, where they live in local arrays of IMPLSCH
 * (wam_source_module.f90:440-462); they let a test compare them one by one
 * with another implementation.  While set, every IMPLSCH launch of the
 * context (wamgpu_implsch_*, wamgpu_step_*) writes, for sea point ij
 * (0-based), decisions[ij + ld*q] with
 *   q = 0  JU, NINT(U10/DELU) clamped to 1..JUMAX (source:498),
 *   q = 1  MIJ of the first FRCUTINDEX call (source:563; ST6 :5447-5515),
 *   q = 2  MIJ of the last call, after the update (source:697),
 *   q = 3  LFACTOR iterations (ST6, source:4647-4672; 0 when the stress
 *          needs no reduction, -1 for ST4);
 * and, when llws is not NULL, llws[ij + ld*(b + KL*ML*q)] for bin
 * b = (K-1) + KL*(M-1): the LLWS mask of the first (q = 0) and of the last
 * (q = 1) SINPUT call.  Device pointers of the context's device; ld >= NSEA.
 * decisions = NULL switches the diagnostics off.  The production step
 * writes none of this. */
WAMGPU_API int wamgpu_set_diagnostics(wamgpu_ctx* ctx, int* decisions, unsigned char* llws, int ld);

/* Restart files from and to device buffers: SAVE_RESTART_FILE
 * (wam_restart_module.f90:414-591) and CONNECT_RESTART (:109-327) in the
 * reference's sequential unformatted layout (4-byte record lengths around
 * each record; REAL = 4-byte float on file whatever the context's
 * precision):
 *   record 1   NSEA, CDTPRO, CDTSOU, CDA, CDTA, CDCA (CHARACTER(14) each)
 *   records    U10, UDIR, TAUW (NSEA values each), FL3 (NSEA x KL x ML)
 *   then       DEPTH if CDTA is not blank, U and V (one record) if CDCA is
 *              not blank.
 * ij2newij (host, NSEA 1-based) renumbers as the reference does without the
 * spatial decomposition: file position p holds model point ij2newij[p-1];
 * NULL is the identity (L_DECOMP).  The spectrum moves through a pinned
 * staging buffer in chunks, gathered / scattered on the device, so it is
 * never held whole on the host.  Device buffers in the context's precision;
 * fl3 with leading dimension ld; depth, u, v may be NULL when their dates are
 * blank.  The context must cover the whole grid (no owned range), and the
 * spectrum record must stay below 2 GiB (NSEA*KL*ML*4 bytes).  Reading
 * checks NSEA and every record length against the model grid and returns
 * WAMGPU_E_ARG where the reference calls ABORT1.  Both calls synchronise
 * the context stream; make the buffers' producers finish first. */
typedef struct wamgpu_restart_dates {
  char cdtpro[14], cdtsou[14], cda[14], cdta[14], cdca[14];  /* blank-padded, no terminator */
} wamgpu_restart_dates;
WAMGPU_API int wamgpu_restart_write(wamgpu_ctx* ctx, const char* path, const void* fl3, int ld, const void* u10,
                                    const void* udir, const void* tauw, const void* depth, const void* u,
                                    const void* v, const wamgpu_restart_dates* dates, const int* ij2newij);
WAMGPU_API int wamgpu_restart_read(wamgpu_ctx* ctx, const char* path, void* fl3, int ld, void* u10, void* udir,
                                   void* tauw, void* depth, void* u, void* v, wamgpu_restart_dates* dates,
                                   const int* ij2newij);

/* New wind fields on the device: GET_WIND's conversion of an input field
 * to the sea points (WAM_WIND, wam_wind_module.f90:1063-1216), so that a
 * pass with hourly winds keeps U10 and UDIR resident.
 *  - wamgpu_set_wind_grid: INITIALIZE of INTERPOLATION_TO_GRID (:1296-1375)
 *    for the input grid of nx_in x ny_in points with west/south corner and
 *    steps in the reference's integer units (1/100 arc-second, M_SEC),
 *    periodic in longitude or not, from the model grid's AMOWEP, AMOSOP,
 *    XDELLA, ZDELLO (one per latitude row) and IFROMIJ (one per sea point;
 *    KFROMIJ is the context's).  equal_grid != 0: the input grid is the
 *    model grid (EQUAL_GRID), and point (IFROMIJ, KFROMIJ) is copied.  A sea
 *    point outside the input grid is WAMGPU_E_ARG, where the reference calls
 *    ABORT1.
 *  - wamgpu_wind_dev: u_in, v_in (device, nx_in x ny_in, longitude fastest)
 *    of WIND CODE code_in (1 friction velocity, 2 surface stress, 3 U10) to
 *    U10 >= 2 m/s and UDIR = ATAN2(U,V) in [0, 2*pi) at every sea point of the
 *    context, in its precision. */
WAMGPU_API int wamgpu_set_wind_grid(wamgpu_ctx* ctx, int nx_in, int ny_in, int west_in, int south_in, int dx_in,
                                    int dy_in, int periodic, int equal_grid, int amowep, int amosop, int xdella,
                                    const int* zdello, const int* ifromij);
WAMGPU_API int wamgpu_wind_dev(wamgpu_ctx* ctx, const void* u_in, const void* v_in, int code_in, void* u10, void* udir,
                               void* stream);

/* PUT_ICE (FL3, INDICATOR) and PUT_DRY (FL3, INDICATOR) on device data
 * (PUT_ICE_SPEC wam_ice_module.f90:312-324, PUT_DRY_SPEC
 * wam_topo_module.f90:557-569; called by WAMODEL at wamodel.f90:380-397),
 * and their parameter-block forms PUT_ICE_PAR / PUT_DRY_PAR (:283-308,
 * :529-553).  data holds nrows rows of ld values with the sea point fastest
 * (a spectrum: nrows = KL*ML; an output block: one row per parameter);
 * points is a device array of n 1-based sea point numbers (IJ_ICE, IJ_DRY).
 * Every row of every listed point becomes `value` (converted to the
 * context's precision); points outside the owned range are skipped, as the
 * reference skips those outside NIJS..NIJL.  This keeps a WAMODEL pass with
 * ice or dry points on the device. */
WAMGPU_API int wamgpu_put_points_dev(wamgpu_ctx* ctx, void* data, int ld, int nrows, const int* points, int n,
                                     double value, void* stream);

/* COMPUTE_OUTPUT_PARAMETER (wam_output_module.f90:481-640) on the device:
 * the integrated parameters of every owned sea point from the resident
 * spectrum, so that an output step reads WAMGPU_OUT_NPARAM values per point
 * instead of the whole spectrum.  block[ij + block_ld*(IP-1)] receives the
 * reference's output parameter IP (CFLAG_P numbering):
 *   1 U10 [m/s], 2 wind direction [deg], 3 USTAR [m/s], 4 drag coefficient,
 *   5 Charnock parameter (CHARNOCK_PAR, wam_interface_module.f90:159),
 *   6 water depth [m] (999 in deep water), 7 current speed [m/s],
 *   8 current direction [deg], 9 significant wave height Hs [m]
 *   (TOTAL_ENERGY :1342), 10 peak period [s] (PEAK_PERIOD :741),
 *   11 mean period 1/FM [s] (FEMEAN :207), 12 TM1 and 13 TM2 [s]
 *   (TM1_TM2_PERIODS :1152), 14 mean direction and 15 directional spread
 *   [deg] (MEAN_DIRECTION :412), 16 normalised wave stress, 32 Z0 [m],
 *   40 mean square slope (MEANSQS :639).
 * The other parameters up to WAMGPU_OUT_NPARAM are set to 0: the wind-sea
 * and swell parameters 17-23 and 25-31 come from wamgpu_output_swell_dev;
 * kurtosis (33-39) is not computed.
 * from != 0 gives directions the waves and wind come from (the reference's
 * default orientation_of_directions), 0 directions they go to.  When USTAR
 * is zero at every point, AIRSEA (wam_source_module.f90:868-971) first sets
 * USTAR and Z0 from U10 and TAUW, as the reference does.  Device pointers in
 * the context's precision, spectrum and fields as for wamgpu_implsch_dev;
 * currents and depth are the context's own. */
#define WAMGPU_OUT_NPARAM 40
WAMGPU_API int wamgpu_output_parameters_dev(wamgpu_ctx* ctx, const void* fl3, int ld, const void* u10,
                                            const void* udir, const void* tauw, void* ustar, void* z0, int from,
                                            void* block, int block_ld, void* stream);

/* SWELL_SEPARATION (wam_swell_module.f90:106-350, called by
 * COMPUTE_OUTPUT_PARAMETER at wam_output_module.f90:637) on the device: the
 * wind-sea parameters 17-23 and the swell parameters 25-31 of the block
 * (significant wave height, peak period, mean period, TM1, TM2, mean
 * direction, directional spread), the other rows untouched.  A bin is swell
 * where 28/C(M) * 1.2*USTAR*COS(TH(K)-UDIR) < 1.  The swell partitioning
 * (parameters 41-49) is not computed.  ustar is the USTAR of the step (after
 * wamgpu_output_parameters_dev when that set it); from as there. */
WAMGPU_API int wamgpu_output_swell_dev(wamgpu_ctx* ctx, const void* fl3, int ld, const void* udir, const void* ustar,
                                       int from, void* block, int block_ld, void* stream);

/* Synchronises the context stream; returns WAMGPU_E_NUMERIC if a kernel
 * reported non-finite output since the last call. */
WAMGPU_API int wamgpu_sync(wamgpu_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* WAMGPU_H */
