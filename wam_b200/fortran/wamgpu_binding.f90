! ISO_C_BINDING shim between WAM Cycle 7 (myWAveModel/WAM) and libwamgpu.
!
! WAMGPU_BINDING declares the C entry points of include/wamgpu.h.
! WAM_GPU_SOURCE_PROPAGATION gives the reference's own procedure names and
! argument lists (IMPLSCH wam_source_module.f90:374, PROPAGS
! wam_propagation_module.f90:635, PREPARE_PROPAGATION :279,
! MAKE_SHALLOW_SNL source:975, PUT_ICE wam_ice_module.f90:312, PUT_DRY
! wam_topo_module.f90:557), so that WAMODEL (src/chief/wamodel.f90) and
! INITMDL compile against it with a changed USE line.  WAM_GPU_DRIVER holds
! the device-resident form of one PROP iteration of WAMODEL
! (wamodel.f90:286-451): the spectrum stays on the GPU across the PROP and
! PHYSICS loops, ice and dry points are zeroed there, and only the
! integrated output parameters come back at output times.
!
! Errors: every call returns 0 or a negative WAMGPU_E* code; WAMGPU_CHECK
! writes wamgpu_last_error to IU06 and calls ABORT1, as the reference does on
! its own errors.
MODULE WAMGPU_BINDING
   USE, INTRINSIC :: ISO_C_BINDING
   IMPLICIT NONE

   TYPE, BIND(C) :: WAMGPU_CONFIG          ! struct wamgpu_config
      INTEGER(C_INT)  :: KL, ML
      REAL(C_DOUBLE)  :: FR1
      INTEGER(C_INT)  :: IREF, IPHYS
      INTEGER(C_INT)  :: SHALLOW_RUN, SPHERICAL_RUN, REFRACTION_D_RUN, REFRACTION_C_RUN, REDUCED_GRID
      INTEGER(C_INT)  :: ISNONLIN, LCFLX
      INTEGER(C_INT)  :: IDELT, IDELPRO
      REAL(C_DOUBLE)  :: BETAMAX, ZALP, ALPHA, TAUWSHELTER, CDFAC
      INTEGER(C_INT)  :: NDEPTH
      REAL(C_DOUBLE)  :: DEPTHA, DEPTHD, DELPHI
      INTEGER(C_INT)  :: PRECISION, DEVICE
   END TYPE WAMGPU_CONFIG

   INTEGER(C_INT), PARAMETER :: WAMGPU_OUT_NPARAM = 40

   INTERFACE
      INTEGER(C_INT) FUNCTION wamgpu_create(cfg, ctx) BIND(C, NAME='wamgpu_create')
         IMPORT :: C_INT, C_PTR, WAMGPU_CONFIG
         TYPE(WAMGPU_CONFIG), INTENT(IN) :: cfg
         TYPE(C_PTR), INTENT(OUT)        :: ctx
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_destroy(ctx) BIND(C, NAME='wamgpu_destroy')
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_config_size() BIND(C, NAME='wamgpu_config_size')
         IMPORT :: C_INT
      END FUNCTION
      TYPE(C_PTR) FUNCTION wamgpu_last_error(ctx) BIND(C, NAME='wamgpu_last_error')
         IMPORT :: C_PTR
         TYPE(C_PTR), VALUE :: ctx
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_set_grid(ctx, nsea, klat, klon, wlat, kfromij, ny, sinph, cosph, dellam) &
&                    BIND(C, NAME='wamgpu_set_grid')
         IMPORT :: C_INT, C_FLOAT, C_PTR
         TYPE(C_PTR), VALUE    :: ctx
         INTEGER(C_INT), VALUE :: nsea, ny
         INTEGER(C_INT)        :: klat(*), klon(*), kfromij(*)
         REAL(C_FLOAT)         :: wlat(*), sinph(*), cosph(*), dellam(*)
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_set_depth(ctx, depth) BIND(C, NAME='wamgpu_set_depth')
         IMPORT :: C_INT, C_FLOAT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         REAL(C_FLOAT)      :: depth(*)
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_set_current(ctx, u, v) BIND(C, NAME='wamgpu_set_current')
         IMPORT :: C_INT, C_FLOAT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         REAL(C_FLOAT)      :: u(*), v(*)
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_prepare_propagation(ctx, total_cfl, counter) &
&                    BIND(C, NAME='wamgpu_prepare_propagation')
         IMPORT :: C_INT, C_FLOAT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         REAL(C_FLOAT)      :: total_cfl
         INTEGER(C_INT)     :: counter
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_prepare_source(ctx) BIND(C, NAME='wamgpu_prepare_source')
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_implsch_host(ctx, fl3, u10, udir, tauw, ustar, z0, roairn, wstar, depth, indep) &
&                    BIND(C, NAME='wamgpu_implsch_host')
         IMPORT :: C_INT, C_FLOAT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         REAL(C_FLOAT)      :: fl3(*), u10(*), udir(*), tauw(*), ustar(*), z0(*), roairn(*), wstar(*), depth(*)
         INTEGER(C_INT)     :: indep(*)
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_propags_host(ctx, f3) BIND(C, NAME='wamgpu_propags_host')
         IMPORT :: C_INT, C_FLOAT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         REAL(C_FLOAT)      :: f3(*)
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_step_host(ctx, fl3, nprop, u10, udir, tauw, ustar, z0, roairn, wstar) &
&                    BIND(C, NAME='wamgpu_step_host')
         IMPORT :: C_INT, C_FLOAT, C_PTR
         TYPE(C_PTR), VALUE    :: ctx
         INTEGER(C_INT), VALUE :: nprop
         REAL(C_FLOAT)         :: fl3(*), u10(*), udir(*), tauw(*), ustar(*), z0(*), roairn(*), wstar(*)
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_step_dev(ctx, fl3, ld, scratch, nprop, u10, udir, tauw, ustar, z0, roairn, &
&                    wstar, stream) BIND(C, NAME='wamgpu_step_dev')
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE    :: ctx, fl3, scratch, u10, udir, tauw, ustar, z0, roairn, wstar, stream
         INTEGER(C_INT), VALUE :: ld, nprop
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_put_points_dev(ctx, data, ld, nrows, points, n, val, stream) &
&                    BIND(C, NAME='wamgpu_put_points_dev')
         IMPORT :: C_INT, C_DOUBLE, C_PTR
         TYPE(C_PTR), VALUE    :: ctx, data, points, stream
         INTEGER(C_INT), VALUE :: ld, nrows, n
         REAL(C_DOUBLE), VALUE :: val
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_output_parameters_dev(ctx, fl3, ld, u10, udir, tauw, ustar, z0, from, &
&                    block, block_ld, stream) BIND(C, NAME='wamgpu_output_parameters_dev')
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE    :: ctx, fl3, u10, udir, tauw, ustar, z0, block, stream
         INTEGER(C_INT), VALUE :: ld, from, block_ld
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_output_swell_dev(ctx, fl3, ld, udir, ustar, from, block, block_ld, stream) &
&                    BIND(C, NAME='wamgpu_output_swell_dev')
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE    :: ctx, fl3, udir, ustar, block, stream
         INTEGER(C_INT), VALUE :: ld, from, block_ld
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_get_fluxes(ctx, out7) BIND(C, NAME='wamgpu_get_fluxes')
         IMPORT :: C_INT, C_FLOAT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
         REAL(C_FLOAT)      :: out7(*)
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_set_owned(ctx, i0, i1) BIND(C, NAME='wamgpu_set_owned')
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE    :: ctx
         INTEGER(C_INT), VALUE :: i0, i1
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_set_counter(ctx, counter) BIND(C, NAME='wamgpu_set_counter')
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE    :: ctx
         INTEGER(C_INT), VALUE :: counter
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_propags_substep_dev(ctx, src, dst, ld, stream) &
&                    BIND(C, NAME='wamgpu_propags_substep_dev')
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE    :: ctx, src, dst, stream
         INTEGER(C_INT), VALUE :: ld
      END FUNCTION
      INTEGER(C_INT) FUNCTION wamgpu_sync(ctx) BIND(C, NAME='wamgpu_sync')
         IMPORT :: C_INT, C_PTR
         TYPE(C_PTR), VALUE :: ctx
      END FUNCTION
   END INTERFACE

   TYPE(C_PTR), SAVE :: CTX = C_NULL_PTR

CONTAINS

   SUBROUTINE WAMGPU_CHECK (RC, WHERE)
      USE WAM_GENERAL_MODULE, ONLY: ABORT1
      USE WAM_FILE_MODULE,    ONLY: IU06
      INTEGER(C_INT),   INTENT(IN) :: RC
      CHARACTER(LEN=*), INTENT(IN) :: WHERE
      CHARACTER(KIND=C_CHAR), POINTER :: MSG(:)
      INTEGER :: N
      IF (RC == 0) RETURN
      CALL C_F_POINTER (wamgpu_last_error(CTX), MSG, [512])
      N = 0
      DO WHILE (N < 512)
         IF (MSG(N+1) == C_NULL_CHAR) EXIT
         N = N + 1
      END DO
      WRITE (IU06,*) ' *** libwamgpu error in ', WHERE, ' (', RC, '): ', MSG(1:N)
      CALL ABORT1
   END SUBROUTINE WAMGPU_CHECK

END MODULE WAMGPU_BINDING

! The reference's procedure names on host arrays (drop-in for the modules'
! procedures; the spectrum goes up and down on every call).
MODULE WAM_GPU_SOURCE_PROPAGATION
   USE WAMGPU_BINDING
   IMPLICIT NONE
   PRIVATE
   PUBLIC :: IMPLSCH, PROPAGS, PUT_ICE_GPU, PUT_DRY_GPU
CONTAINS
   SUBROUTINE IMPLSCH (FL3, U10, UDIR, TAUW, USTAR, Z0, ROAIRN, WSTAR, DEPTH, INDEP)
      REAL,    INTENT(INOUT), TARGET :: FL3(:,:,:), TAUW(:), USTAR(:), Z0(:)
      REAL,    INTENT(IN),    TARGET :: U10(:), UDIR(:), ROAIRN(:), WSTAR(:), DEPTH(:)
      INTEGER, INTENT(IN),    TARGET :: INDEP(:)
      CALL WAMGPU_CHECK (wamgpu_implsch_host(CTX, FL3, U10, UDIR, TAUW, USTAR, Z0, ROAIRN, WSTAR, &
&                        DEPTH, INDEP), 'IMPLSCH')
   END SUBROUTINE IMPLSCH

   SUBROUTINE PROPAGS (F3)
      REAL, INTENT(INOUT), TARGET :: F3(:,:,:)
      CALL WAMGPU_CHECK (wamgpu_propags_host(CTX, F3), 'PROPAGS')
   END SUBROUTINE PROPAGS

   ! PUT_ICE (FL3, INDICATOR) / PUT_DRY (FL3, INDICATOR) on the resident
   ! device spectrum FL3_DEV (leading dimension LD): IJ_DEV is a device copy of
   ! IJ_ICE / IJ_DRY (N entries, 1-based sea points).
   SUBROUTINE PUT_ICE_GPU (FL3_DEV, LD, NBINS, IJ_DEV, N, INDICATOR)
      TYPE(C_PTR), INTENT(IN) :: FL3_DEV, IJ_DEV
      INTEGER,     INTENT(IN) :: LD, NBINS, N
      REAL,        INTENT(IN) :: INDICATOR
      CALL WAMGPU_CHECK (wamgpu_put_points_dev(CTX, FL3_DEV, INT(LD, C_INT), INT(NBINS, C_INT), IJ_DEV,  &
&                        INT(N, C_INT), REAL(INDICATOR, C_DOUBLE), C_NULL_PTR), 'PUT_ICE')
   END SUBROUTINE PUT_ICE_GPU

   SUBROUTINE PUT_DRY_GPU (FL3_DEV, LD, NBINS, IJ_DEV, N, INDICATOR)
      TYPE(C_PTR), INTENT(IN) :: FL3_DEV, IJ_DEV
      INTEGER,     INTENT(IN) :: LD, NBINS, N
      REAL,        INTENT(IN) :: INDICATOR
      CALL WAMGPU_CHECK (wamgpu_put_points_dev(CTX, FL3_DEV, INT(LD, C_INT), INT(NBINS, C_INT), IJ_DEV,  &
&                        INT(N, C_INT), REAL(INDICATOR, C_DOUBLE), C_NULL_PTR), 'PUT_DRY')
   END SUBROUTINE PUT_DRY_GPU
END MODULE WAM_GPU_SOURCE_PROPAGATION

! One PROP iteration of WAMODEL (wamodel.f90:286-451) with the model state
! resident on the device: IDELT/IDELPRO propagation steps and the source
! step (wamgpu_step_dev), then PUT_ICE and PUT_DRY (:380-397), and, at output
! times, the integrated parameters of COMPUTE_OUTPUT_PARAMETER
! (wam_output_module.f90:481-640) copied back (NSEA x WAMGPU_OUT_NPARAM
! values instead of the spectrum).  The device buffers are the driver's own
! (cudaMalloc'd or OpenACC data regions) and are passed as C pointers.
MODULE WAM_GPU_DRIVER
   USE WAMGPU_BINDING
   IMPLICIT NONE
   PRIVATE
   PUBLIC :: WAMGPU_PASS, WAMGPU_OUTPUT

   TYPE, PUBLIC :: WAMGPU_STATE
      TYPE(C_PTR) :: FL3 = C_NULL_PTR, SCRATCH = C_NULL_PTR
      TYPE(C_PTR) :: U10 = C_NULL_PTR, UDIR = C_NULL_PTR, TAUW = C_NULL_PTR, USTAR = C_NULL_PTR
      TYPE(C_PTR) :: Z0 = C_NULL_PTR, ROAIRN = C_NULL_PTR, WSTAR = C_NULL_PTR
      TYPE(C_PTR) :: IJ_ICE = C_NULL_PTR, IJ_DRY = C_NULL_PTR, BLOCK = C_NULL_PTR
      INTEGER     :: LD = 0, NBINS = 0, N_ICE = 0, N_DRY = 0
   END TYPE WAMGPU_STATE

CONTAINS

   SUBROUTINE WAMGPU_PASS (S, NPROP, ICE_RUN, SHALLOW_RUN)
      TYPE(WAMGPU_STATE), INTENT(IN) :: S
      INTEGER,            INTENT(IN) :: NPROP
      LOGICAL,            INTENT(IN) :: ICE_RUN, SHALLOW_RUN
      CALL WAMGPU_CHECK (wamgpu_step_dev(CTX, S%FL3, INT(S%LD, C_INT), S%SCRATCH, INT(NPROP, C_INT), S%U10,  &
&                        S%UDIR, S%TAUW, S%USTAR, S%Z0, S%ROAIRN, S%WSTAR, C_NULL_PTR), 'PROP/PHYSICS')
      IF (ICE_RUN .AND. S%N_ICE > 0) THEN
         CALL WAMGPU_CHECK (wamgpu_put_points_dev(CTX, S%FL3, INT(S%LD, C_INT), INT(S%NBINS, C_INT), S%IJ_ICE, &
&                           INT(S%N_ICE, C_INT), 0.0_C_DOUBLE, C_NULL_PTR), 'PUT_ICE')
      END IF
      IF (SHALLOW_RUN .AND. S%N_DRY > 0) THEN
         CALL WAMGPU_CHECK (wamgpu_put_points_dev(CTX, S%FL3, INT(S%LD, C_INT), INT(S%NBINS, C_INT), S%IJ_DRY, &
&                           INT(S%N_DRY, C_INT), 0.0_C_DOUBLE, C_NULL_PTR), 'PUT_DRY')
      END IF
   END SUBROUTINE WAMGPU_PASS

   ! BLOCK of COMPUTE_OUTPUT_PARAMETER into S%BLOCK on the device (leading
   ! dimension S%LD); the driver copies the parameters it writes back.
   SUBROUTINE WAMGPU_OUTPUT (S, FROM)
      TYPE(WAMGPU_STATE), INTENT(IN) :: S
      LOGICAL,            INTENT(IN) :: FROM   ! orientation_of_directions
      INTEGER(C_INT) :: IFROM
      IFROM = 0
      IF (FROM) IFROM = 1
      CALL WAMGPU_CHECK (wamgpu_output_parameters_dev(CTX, S%FL3, INT(S%LD, C_INT), S%U10, S%UDIR, S%TAUW,  &
&                        S%USTAR, S%Z0, IFROM, S%BLOCK, INT(S%LD, C_INT), C_NULL_PTR), 'COMPUTE_OUTPUT_PARAMETER')
      CALL WAMGPU_CHECK (wamgpu_output_swell_dev(CTX, S%FL3, INT(S%LD, C_INT), S%UDIR, S%USTAR, IFROM,      &
&                        S%BLOCK, INT(S%LD, C_INT), C_NULL_PTR), 'SWELL_SEPARATION')
      CALL WAMGPU_CHECK (wamgpu_sync(CTX), 'SYNC')
   END SUBROUTINE WAMGPU_OUTPUT
END MODULE WAM_GPU_DRIVER
