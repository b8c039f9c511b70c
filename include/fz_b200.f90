! firtez-dz B200 -- ISO_C_BINDING interface of the C-ABI in fz_b200.h, for the
! FIRTEZ-dz Fortran host (the pattern src/user_fftw3.f90 already uses to bind
! C).  Every entry point of fz_b200.h has an interface here with the same
! argument list; arrays are passed as the reference's own arrays (column-
! major, first index fastest), device buffers and CUDA streams as TYPE(C_PTR)
! by value, optional host arrays as TYPE(C_PTR) by value (C_LOC(array) or
! C_NULL_PTR).  Return values: 0 = OK, < 0 = FZ_ERR_* (FZ_STRERROR).
!
! Call sites in the reference (see the comments beside each group):
!   START_STEP (src/pre_post_duties.f90:59-93)       -> FZ_LINES_PARSE, FZ_CREATE
!   FORWARD3D / FORWARD1D (src/forward.f90:43-306,
!     :857-1029)                                     -> FZ_FORWARD, FZ_FORWARD_RF
!   GET_PERTURBATION (src/get_dmodel.f90:799-803)    -> FZ_LM_PERTURBATION
!   INVERT3D's cycle (src/invert3d.f90:57-178)       -> FZ_INVERT
MODULE FZ_B200
  USE ISO_C_BINDING
  IMPLICIT NONE
  INTEGER(C_INT), PARAMETER :: FZ_ERR_ARG = -1, FZ_ERR_CUDA = -2, FZ_ERR_NOMEM = -3, FZ_ERR_PARSE = -4
  INTEGER(C_INT), PARAMETER :: FZ_ERR_LIMIT = -5, FZ_ERR_STATE = -6
  INTEGER(C_INT), PARAMETER :: FZ_OK = 0, FZ_CHEM_NOCONV = 1, FZ_NAN = 2
  INTEGER(C_INT), PARAMETER :: FZ_HE_NONE = 0, FZ_HE_TOP = 1, FZ_HE_LTAU = 2
  INTEGER(C_INT), PARAMETER :: FZ_ASSIST_TEMP = 1, FZ_ASSIST_PGAS = 2, FZ_ASSIST_BVEC = 4
  INTEGER(C_INT), PARAMETER :: FZ_ASSIST_VLOS = 8, FZ_ASSIST_PROGRESSIVE = 16
  ! one row of lines_database.dat (NREAD_LINES_DATABASE)
  TYPE, BIND(C) :: FZ_LINE
    INTEGER(C_INT32_T) :: NUM, ZN, ION, FLAG, OTR(2), ABO_IERR, PAD
    REAL(C_DOUBLE)     :: L0, LOGGF, EPLOW, ALPHA, SIGMA
    REAL(C_DOUBLE)     :: SL, LL, JL, SU, LU, JU, ELOWLIM, EUPPLIM
  END TYPE
  ! one region of the LINES: section (BLENDSID 0-based, BLENDSDIFF, WAVE_INIT)
  TYPE, BIND(C) :: FZ_REGION
    INTEGER(C_INT32_T) :: NBLEND, LINE(8)
    REAL(C_DOUBLE)     :: WDIF(8)
    INTEGER(C_INT32_T) :: NUMWAVE, PAD
    REAL(C_DOUBLE)     :: WAVE_INI, DLAMBDA
  END TYPE
  ! options of the batched inversion (control-file values: MAXITER, NOISE, ...)
  TYPE, BIND(C) :: FZ_LM_OPTS
    INTEGER(C_INT) :: MAXSTEPS, MAXIT
    REAL(C_DOUBLE) :: DCHI2, SVDTOL, ISIGMA
    REAL(C_FLOAT)  :: WSTK(4)
    INTEGER(C_INT) :: SLOTS, ASSIST                ! ASSIST: FZ_ASSIST_* bits
    REAL(C_DOUBLE) :: FALLBACK
    TYPE(C_PTR)    :: FALLBACK_MODEL
    INTEGER(C_INT) :: REG_TYPE(8)                  ! PEN_TYP
    REAL(C_DOUBLE) :: REG_ALPHA(8)                 ! PEN_ALP
    INTEGER(C_INT) :: FALLBACK_STEPS
    INTEGER(C_INT) :: SOLVER                       ! SOLVER_METHOD: 1 SVD, 2 CG
    INTEGER(C_INT) :: NODE_EXPANSION               ! 1 SIR-like, 2 STiC-like
    INTEGER(C_INT) :: GLOBAL_STOP                  ! MAKE_DECISION's field rule
    INTEGER(C_INT) :: CYCLES_LEFT                  ! MAXITER - CURIC
    INTEGER(C_INT) :: FALLBACK_FREE                ! the restarted search ignores the goal
    TYPE(C_PTR)    :: STATE_OUT                    ! INV_SLA(1:4), INV_SLA(9) per pixel, or C_NULL_PTR
  END TYPE
  ! launch shapes of the autotuner
  TYPE, BIND(C) :: FZ_TUNE
    INTEGER(C_INT) :: CHAIN_WARPS, CHEMDER_BLOCKS_PER_SM, OPAC_RF_THREADS, LM_SLOTS
    REAL(C_FLOAT)  :: CHAIN_MS, CHEMDER_MS, OPAC_RF_MS, LM_PIXELS_PER_S
    INTEGER(C_INT) :: CHAIN_LANES, PAD
  END TYPE
  INTERFACE
    INTEGER(C_INT) FUNCTION FZ_VERSION() BIND(C, NAME='fz_version')
      IMPORT
    END FUNCTION
    TYPE(C_PTR) FUNCTION FZ_STRERROR(CODE) BIND(C, NAME='fz_strerror')
      IMPORT
      INTEGER(C_INT), VALUE      :: CODE
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LINES_PARSE(TEXT, OUT, MAXN) BIND(C, NAME='fz_lines_parse')
      IMPORT
      CHARACTER(KIND=C_CHAR)     :: TEXT(*)                ! NUL-terminated lines_database.dat text
      TYPE(FZ_LINE)              :: OUT(*)
      INTEGER(C_INT), VALUE      :: MAXN
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_CREATE(CTX, LINES, NLINES, REGIONS, NREGIONS, NZ, GAIN, DEVICE) &
        BIND(C, NAME='fz_create')
      IMPORT
      TYPE(C_PTR)                :: CTX
      TYPE(FZ_LINE)              :: LINES(*)
      INTEGER(C_INT), VALUE      :: NLINES
      TYPE(FZ_REGION)            :: REGIONS(*)
      INTEGER(C_INT), VALUE      :: NREGIONS
      INTEGER(C_INT), VALUE      :: NZ
      TYPE(C_PTR), VALUE         :: GAIN                   ! GAIN1D(4,NUMW)
      INTEGER(C_INT), VALUE      :: DEVICE
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_DESTROY(CTX) BIND(C, NAME='fz_destroy')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_NUMW(CTX) BIND(C, NAME='fz_numw')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_GET_GAIN(CTX, GAIN) BIND(C, NAME='fz_get_gain')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      REAL(C_FLOAT)              :: GAIN(*)                ! GAIN1D(4,NUMW)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_FORWARD(CTX, NCOL, MODEL, HYDROSTATIC, SYN, MODEL_OUT, STATUS) &
        BIND(C, NAME='fz_forward')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      REAL(C_FLOAT)              :: MODEL(*)               ! MODEL(NZ,13,NCOL)
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      REAL(C_DOUBLE)             :: SYN(*)                 ! RSYN1D(NFREQ,NCOL)
      REAL(C_FLOAT)              :: MODEL_OUT(*)           ! MODEL(NZ,13,NCOL), may be MODEL
      INTEGER(C_INT)             :: STATUS(*)              ! per column / pixel
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_FORWARD_DEVICE(CTX, NCOL, D_MODEL, HYDROSTATIC, D_SYN, &
        D_MODEL_OUT, D_STATUS, STREAM) BIND(C, NAME='fz_forward_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      TYPE(C_PTR), VALUE         :: D_MODEL
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(C_PTR), VALUE         :: D_SYN
      TYPE(C_PTR), VALUE         :: D_MODEL_OUT
      TYPE(C_PTR), VALUE         :: D_STATUS
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_FORWARD_DEVICE_STATIC(CTX, NCOL, D_MODEL, HYDROSTATIC, D_SYN, &
        D_MODEL_OUT, D_STATUS, STREAM) BIND(C, NAME='fz_forward_device_static')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      TYPE(C_PTR), VALUE         :: D_MODEL
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(C_PTR), VALUE         :: D_SYN
      TYPE(C_PTR), VALUE         :: D_MODEL_OUT
      TYPE(C_PTR), VALUE         :: D_STATUS
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_HYDROSTATIC(CTX, NCOL, MODEL, HYDROSTATIC, MODEL_OUT, STATUS) &
        BIND(C, NAME='fz_hydrostatic')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      REAL(C_FLOAT)              :: MODEL(*)               ! MODEL(NZ,13,NCOL)
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      REAL(C_FLOAT)              :: MODEL_OUT(*)           ! MODEL(NZ,13,NCOL), may be MODEL
      INTEGER(C_INT)             :: STATUS(*)              ! per column / pixel
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_HYDROSTATIC_DEVICE(CTX, NCOL, D_MODEL, HYDROSTATIC, D_MODEL_OUT, &
        D_STATUS, STREAM) BIND(C, NAME='fz_hydrostatic_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      TYPE(C_PTR), VALUE         :: D_MODEL
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(C_PTR), VALUE         :: D_MODEL_OUT
      TYPE(C_PTR), VALUE         :: D_STATUS
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LOG_TAU5(CTX, NCOL, MODEL, HYDROSTATIC, MODEL_OUT, STATUS) &
        BIND(C, NAME='fz_log_tau5')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      REAL(C_FLOAT)              :: MODEL(*)               ! MODEL(NZ,13,NCOL)
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      REAL(C_FLOAT)              :: MODEL_OUT(*)           ! MODEL(NZ,13,NCOL), may be MODEL
      INTEGER(C_INT)             :: STATUS(*)              ! per column / pixel
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LOG_TAU5_DEVICE(CTX, NCOL, D_MODEL, HYDROSTATIC, D_MODEL_OUT, &
        D_STATUS, STREAM) BIND(C, NAME='fz_log_tau5_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      TYPE(C_PTR), VALUE         :: D_MODEL
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(C_PTR), VALUE         :: D_MODEL_OUT
      TYPE(C_PTR), VALUE         :: D_STATUS
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_RF_NODES(CTX, NODES) BIND(C, NAME='fz_rf_nodes')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT)             :: NODES(*)               ! NJ of T, Pg, rho, Bx, By, Bz, v, P0
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_FORWARD_RF(CTX, NCOL, MODEL, HYDROSTATIC, SYN, JAC, MODEL_OUT, &
        STATUS) BIND(C, NAME='fz_forward_rf')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      REAL(C_FLOAT)              :: MODEL(*)               ! MODEL(NZ,13,NCOL)
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      REAL(C_DOUBLE)             :: SYN(*)                 ! RSYN1D(NFREQ,NCOL)
      REAL(C_FLOAT)              :: JAC(*)                 ! (NF,NP,NPIX)
      REAL(C_FLOAT)              :: MODEL_OUT(*)           ! MODEL(NZ,13,NCOL), may be MODEL
      INTEGER(C_INT)             :: STATUS(*)              ! per column / pixel
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_FORWARD_RF_DEVICE(CTX, NCOL, D_MODEL, HYDROSTATIC, D_SYN, D_JAC, &
        D_MODEL_OUT, D_STATUS, STREAM) BIND(C, NAME='fz_forward_rf_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      TYPE(C_PTR), VALUE         :: D_MODEL
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(C_PTR), VALUE         :: D_SYN
      TYPE(C_PTR), VALUE         :: D_JAC
      TYPE(C_PTR), VALUE         :: D_MODEL_OUT
      TYPE(C_PTR), VALUE         :: D_STATUS
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_FORWARD_RF_FULL(CTX, NCOL, MODEL, HYDROSTATIC, SYN, RF, &
        MODEL_OUT, STATUS) BIND(C, NAME='fz_forward_rf_full')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      REAL(C_FLOAT)              :: MODEL(*)               ! MODEL(NZ,13,NCOL)
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      REAL(C_DOUBLE)             :: SYN(*)                 ! RSYN1D(NFREQ,NCOL)
      REAL(C_FLOAT)              :: RF(*)                  ! DSYN(NFREQ,6*NZ,NCOL)
      REAL(C_FLOAT)              :: MODEL_OUT(*)           ! MODEL(NZ,13,NCOL), may be MODEL
      INTEGER(C_INT)             :: STATUS(*)              ! per column / pixel
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_FORWARD_RF_FULL_DEVICE(CTX, NCOL, D_MODEL, HYDROSTATIC, D_SYN, &
        D_RF, D_MODEL_OUT, D_STATUS, STREAM) BIND(C, NAME='fz_forward_rf_full_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      TYPE(C_PTR), VALUE         :: D_MODEL
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(C_PTR), VALUE         :: D_SYN
      TYPE(C_PTR), VALUE         :: D_RF
      TYPE(C_PTR), VALUE         :: D_MODEL_OUT
      TYPE(C_PTR), VALUE         :: D_STATUS
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_AUTOTUNE_FORWARD(CTX, NCOL, D_MODEL, HYDROSTATIC, OUT) BIND(C, &
        NAME='fz_autotune_forward')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NCOL
      TYPE(C_PTR), VALUE         :: D_MODEL
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(FZ_TUNE)              :: OUT
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_TUNE_GET(CTX, OUT) BIND(C, NAME='fz_tune_get')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      TYPE(FZ_TUNE)              :: OUT
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_TUNE_SET(CTX, T) BIND(C, NAME='fz_tune_set')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      TYPE(FZ_TUNE)              :: T
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_SMOOTH(CTX, NX, NY, MODELS, PARAMS) BIND(C, NAME='fz_smooth')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      REAL(C_FLOAT)              :: MODELS(*)              ! MODEL(NZ,13,NPIX)
      TYPE(C_PTR), VALUE         :: PARAMS                 ! 1 = smooth T..P0, or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_SMOOTH_DEVICE(CTX, NX, NY, D_MODELS, PARAMS, STREAM) BIND(C, &
        NAME='fz_smooth_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      TYPE(C_PTR), VALUE         :: D_MODELS
      TYPE(C_PTR), VALUE         :: PARAMS                 ! 1 = smooth T..P0, or C_NULL_PTR
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_INVERT(CTX, NPIX, OBS, INIT, TARGET_CHI2, HYDROSTATIC, OPTS, &
        MODEL_OUT, CHI2, ITERS, SYN_OUT, STATUS) BIND(C, NAME='fz_invert')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NPIX
      REAL(C_DOUBLE)             :: OBS(*)                 ! OBS3D(NFREQ,NPIX)
      REAL(C_FLOAT)              :: INIT(*)                ! MODEL(NZ,13,NPIX)
      TYPE(C_PTR), VALUE         :: TARGET_CHI2            ! per-pixel chi2 goal or C_NULL_PTR
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(FZ_LM_OPTS)           :: OPTS
      REAL(C_FLOAT)              :: MODEL_OUT(*)           ! MODEL(NZ,13,NCOL), may be MODEL
      REAL(C_DOUBLE)             :: CHI2(*)
      INTEGER(C_INT)             :: ITERS(*)
      TYPE(C_PTR), VALUE         :: SYN_OUT                ! RSYN1D(NFREQ,NPIX) or C_NULL_PTR
      INTEGER(C_INT)             :: STATUS(*)              ! per column / pixel
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_INVERT_DEVICE(CTX, NPIX, D_OBS, D_INIT, D_TARGET_CHI2, &
        HYDROSTATIC, OPTS, D_MODEL_OUT, D_CHI2, D_ITERS, D_SYN_OUT, D_STATUS, STREAM) BIND(C, &
        NAME='fz_invert_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NPIX
      TYPE(C_PTR), VALUE         :: D_OBS
      TYPE(C_PTR), VALUE         :: D_INIT
      TYPE(C_PTR), VALUE         :: D_TARGET_CHI2
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(FZ_LM_OPTS)           :: OPTS
      TYPE(C_PTR), VALUE         :: D_MODEL_OUT
      TYPE(C_PTR), VALUE         :: D_CHI2
      TYPE(C_PTR), VALUE         :: D_ITERS
      TYPE(C_PTR), VALUE         :: D_SYN_OUT
      TYPE(C_PTR), VALUE         :: D_STATUS
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_AUTOTUNE_LM(CTX, NPIX, D_OBS, D_INIT, D_TARGET_CHI2, HYDROSTATIC, &
        OPTS, CANDIDATES, NCAND, OUT) BIND(C, NAME='fz_autotune_lm')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NPIX
      TYPE(C_PTR), VALUE         :: D_OBS
      TYPE(C_PTR), VALUE         :: D_INIT
      TYPE(C_PTR), VALUE         :: D_TARGET_CHI2
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(FZ_LM_OPTS)           :: OPTS
      INTEGER(C_INT)             :: CANDIDATES(*)
      INTEGER(C_INT), VALUE      :: NCAND
      TYPE(FZ_TUNE)              :: OUT
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_SMOOTH_SHARD_DEVICE(CTX, NX, NY, X0, NX_FIELD, D_MODELS, PARAMS, &
        STREAM) BIND(C, NAME='fz_smooth_shard_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      INTEGER(C_INT), VALUE      :: X0
      INTEGER(C_INT), VALUE      :: NX_FIELD
      TYPE(C_PTR), VALUE         :: D_MODELS
      TYPE(C_PTR), VALUE         :: PARAMS                 ! 1 = smooth T..P0, or C_NULL_PTR
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_INVERT_CYCLES_DEVICE(CTX, NX, NY, D_OBS, D_MODELS, NCYCLES, &
        NODES, HYDROSTATIC, OPTS, D_CHI2, D_ITERS, D_STATUS, STREAM) BIND(C, &
        NAME='fz_invert_cycles_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      TYPE(C_PTR), VALUE         :: D_OBS
      TYPE(C_PTR), VALUE         :: D_MODELS
      INTEGER(C_INT), VALUE      :: NCYCLES
      INTEGER(C_INT)             :: NODES(*)               ! NJ of T, Pg, rho, Bx, By, Bz, v, P0
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(FZ_LM_OPTS)           :: OPTS
      TYPE(C_PTR), VALUE         :: D_CHI2
      TYPE(C_PTR), VALUE         :: D_ITERS
      TYPE(C_PTR), VALUE         :: D_STATUS
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LSF_GAUSSIAN(CTX, REGION, SIGMA, W0) BIND(C, &
        NAME='fz_lsf_gaussian')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: REGION
      REAL(C_DOUBLE), VALUE      :: SIGMA
      REAL(C_DOUBLE), VALUE      :: W0
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LSF_KERNEL(CTX, REGION, YK, N) BIND(C, NAME='fz_lsf_kernel')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: REGION
      REAL(C_DOUBLE)             :: YK(*)
      INTEGER(C_INT), VALUE      :: N
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LSF_CLEAR(CTX) BIND(C, NAME='fz_lsf_clear')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_SET_TAU_DEVICE(CTX, NX, NY, D_OBS, D_MODELS, ASSIST, HYDROSTATIC, &
        STREAM) BIND(C, NAME='fz_set_tau_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      TYPE(C_PTR), VALUE         :: D_OBS
      TYPE(C_PTR), VALUE         :: D_MODELS
      INTEGER(C_INT), VALUE      :: ASSIST
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_SET_TAU(CTX, NX, NY, OBS, MODELS, ASSIST, HYDROSTATIC) BIND(C, &
        NAME='fz_set_tau')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      REAL(C_DOUBLE)             :: OBS(*)                 ! OBS3D(NFREQ,NPIX)
      REAL(C_FLOAT)              :: MODELS(*)              ! MODEL(NZ,13,NPIX)
      INTEGER(C_INT), VALUE      :: ASSIST
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_SET_TAU_SHARD_DEVICE(CTX, NX, NY, D_OBS, D_MODELS, ASSIST, &
        HYDROSTATIC, REDUCE, USER, STREAM) BIND(C, NAME='fz_set_tau_shard_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      TYPE(C_PTR), VALUE         :: D_OBS
      TYPE(C_PTR), VALUE         :: D_MODELS
      INTEGER(C_INT), VALUE      :: ASSIST
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(C_FUNPTR), VALUE      :: REDUCE
      TYPE(C_PTR), VALUE         :: USER
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_ERRORS_DEVICE(CTX, NPIX, D_OBS, D_MODELS, HYDROSTATIC, OPTS, &
        D_ERR, D_CHI2, D_STATUS, STREAM) BIND(C, NAME='fz_errors_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NPIX
      TYPE(C_PTR), VALUE         :: D_OBS
      TYPE(C_PTR), VALUE         :: D_MODELS
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(FZ_LM_OPTS)           :: OPTS
      TYPE(C_PTR), VALUE         :: D_ERR
      TYPE(C_PTR), VALUE         :: D_CHI2
      TYPE(C_PTR), VALUE         :: D_STATUS
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_ERRORS(CTX, NPIX, OBS, MODELS, HYDROSTATIC, OPTS, ERR, CHI2, &
        STATUS) BIND(C, NAME='fz_errors')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NPIX
      REAL(C_DOUBLE)             :: OBS(*)                 ! OBS3D(NFREQ,NPIX)
      REAL(C_FLOAT)              :: MODELS(*)              ! MODEL(NZ,13,NPIX)
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(FZ_LM_OPTS)           :: OPTS
      REAL(C_FLOAT)              :: ERR(*)
      REAL(C_DOUBLE)             :: CHI2(*)
      INTEGER(C_INT)             :: STATUS(*)              ! per column / pixel
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LM_PERTURBATION(CTX, NPIX, NP, NFREQ, JAC, DIFF, LAMBDA, REG_PEN, &
        REG_HSS, DTYPE, SVDTOL, DELTA) BIND(C, NAME='fz_lm_perturbation')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NPIX
      INTEGER(C_INT), VALUE      :: NP
      INTEGER(C_INT), VALUE      :: NFREQ
      REAL(C_DOUBLE)             :: JAC(*)                 ! (NF,NP,NPIX)
      REAL(C_DOUBLE)             :: DIFF(*)
      REAL(C_DOUBLE)             :: LAMBDA(*)
      TYPE(C_PTR), VALUE         :: REG_PEN                ! PEN_RES(NP,NPIX) or C_NULL_PTR
      TYPE(C_PTR), VALUE         :: REG_HSS                ! PEN_HSS(NP,NP,NPIX) or C_NULL_PTR
      INTEGER(C_INT), VALUE      :: DTYPE
      REAL(C_DOUBLE), VALUE      :: SVDTOL
      REAL(C_DOUBLE)             :: DELTA(*)               ! (NP,NPIX)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LM_PERTURBATION_F32(CTX, NPIX, NP, NFREQ, JAC, DIFF, LAMBDA, &
        REG_PEN, REG_HSS, DTYPE, SVDTOL, DELTA) BIND(C, NAME='fz_lm_perturbation_f32')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NPIX
      INTEGER(C_INT), VALUE      :: NP
      INTEGER(C_INT), VALUE      :: NFREQ
      REAL(C_FLOAT)              :: JAC(*)                 ! (NF,NP,NPIX)
      REAL(C_DOUBLE)             :: DIFF(*)
      REAL(C_DOUBLE)             :: LAMBDA(*)
      TYPE(C_PTR), VALUE         :: REG_PEN                ! PEN_RES(NP,NPIX) or C_NULL_PTR
      TYPE(C_PTR), VALUE         :: REG_HSS                ! PEN_HSS(NP,NP,NPIX) or C_NULL_PTR
      INTEGER(C_INT), VALUE      :: DTYPE
      REAL(C_DOUBLE), VALUE      :: SVDTOL
      REAL(C_DOUBLE)             :: DELTA(*)               ! (NP,NPIX)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LM_UPDATE_LAMBDA(N, CHICUR, CHIPRE, LAMBDA, STEPS, PRECYC) &
        BIND(C, NAME='fz_lm_update_lambda')
      IMPORT
      INTEGER(C_INT), VALUE      :: N
      REAL(C_DOUBLE)             :: CHICUR(*)              ! chi2 of the new models
      REAL(C_DOUBLE)             :: CHIPRE(*)
      REAL(C_DOUBLE)             :: LAMBDA(*)
      REAL(C_DOUBLE)             :: STEPS(*)
      REAL(C_DOUBLE)             :: PRECYC(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LM_UPDATE_LAMBDA_DEVICE(N, D_CHICUR, D_CHIPRE, D_LAMBDA, D_STEPS, &
        D_PRECYC, STREAM) BIND(C, NAME='fz_lm_update_lambda_device')
      IMPORT
      INTEGER(C_INT), VALUE      :: N
      TYPE(C_PTR), VALUE         :: D_CHICUR
      TYPE(C_PTR), VALUE         :: D_CHIPRE
      TYPE(C_PTR), VALUE         :: D_LAMBDA
      TYPE(C_PTR), VALUE         :: D_STEPS
      TYPE(C_PTR), VALUE         :: D_PRECYC
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LM_REARANGE(CTX, NPIX, MODELS, DELTA, NODE_EXPANSION) BIND(C, &
        NAME='fz_lm_rearange')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NPIX
      REAL(C_FLOAT)              :: MODELS(*)              ! MODEL(NZ,13,NPIX)
      REAL(C_DOUBLE)             :: DELTA(*)               ! (NP,NPIX)
      INTEGER(C_INT), VALUE      :: NODE_EXPANSION
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_LM_REARANGE_DEVICE(CTX, NPIX, D_MODELS, D_DELTA, NODE_EXPANSION, &
        STREAM) BIND(C, NAME='fz_lm_rearange_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: NPIX
      TYPE(C_PTR), VALUE         :: D_MODELS
      TYPE(C_PTR), VALUE         :: D_DELTA
      INTEGER(C_INT), VALUE      :: NODE_EXPANSION
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_RTE_SOLVE(NCOL, NZ, NW, ETA, SRC, ZZ, BND, OUT) BIND(C, &
        NAME='fz_rte_solve')
      IMPORT
      INTEGER(C_INT), VALUE      :: NCOL
      INTEGER(C_INT), VALUE      :: NZ
      INTEGER(C_INT), VALUE      :: NW
      REAL(C_FLOAT)              :: ETA(*)                 ! (NW,7,NZ,NCOL) ETAI..RHOV
      REAL(C_FLOAT)              :: SRC(*)
      REAL(C_DOUBLE)             :: ZZ(*)                  ! ZZ(NZ) km
      TYPE(C_PTR), VALUE         :: BND                    ! (NZ,NCOL) boundary flags
      REAL(C_DOUBLE)             :: OUT(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_RTE_SOLVE_DEVICE(NCOL, NZ, NW, D_ETA, D_SRC, D_ZZ, D_BND, D_OUT, &
        STREAM) BIND(C, NAME='fz_rte_solve_device')
      IMPORT
      INTEGER(C_INT), VALUE      :: NCOL
      INTEGER(C_INT), VALUE      :: NZ
      INTEGER(C_INT), VALUE      :: NW
      TYPE(C_PTR), VALUE         :: D_ETA
      TYPE(C_PTR), VALUE         :: D_SRC
      TYPE(C_PTR), VALUE         :: D_ZZ
      TYPE(C_PTR), VALUE         :: D_BND
      TYPE(C_PTR), VALUE         :: D_OUT
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_VOIGT(N, A, V, H, F) BIND(C, NAME='fz_voigt')
      IMPORT
      INTEGER(C_INT), VALUE      :: N
      REAL(C_FLOAT)              :: A(*)
      REAL(C_FLOAT)              :: V(*)
      REAL(C_FLOAT)              :: H(*)
      REAL(C_FLOAT)              :: F(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MLP_CREATE(MLP, NLAYERS, DIMS, SEED, DEVICE) BIND(C, &
        NAME='fz_mlp_create')
      IMPORT
      TYPE(C_PTR)                :: MLP
      INTEGER(C_INT), VALUE      :: NLAYERS
      INTEGER(C_INT)             :: DIMS(*)
      INTEGER(C_LONG_LONG), VALUE :: SEED
      INTEGER(C_INT), VALUE      :: DEVICE
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MLP_DESTROY(MLP) BIND(C, NAME='fz_mlp_destroy')
      IMPORT
      TYPE(C_PTR), VALUE         :: MLP
    END FUNCTION
    INTEGER(C_LONG_LONG) FUNCTION FZ_MLP_NPARAMS(MLP) BIND(C, NAME='fz_mlp_nparams')
      IMPORT
      TYPE(C_PTR), VALUE         :: MLP
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MLP_GET_PARAMS(MLP, HOST, GRADS) BIND(C, &
        NAME='fz_mlp_get_params')
      IMPORT
      TYPE(C_PTR), VALUE         :: MLP
      REAL(C_FLOAT)              :: HOST(*)
      INTEGER(C_INT), VALUE      :: GRADS
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MLP_SET_PARAMS(MLP, HOST) BIND(C, NAME='fz_mlp_set_params')
      IMPORT
      TYPE(C_PTR), VALUE         :: MLP
      REAL(C_FLOAT)              :: HOST(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MLP_FORWARD_DEVICE(MLP, N, D_X, D_Y, STREAM) BIND(C, &
        NAME='fz_mlp_forward_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: MLP
      INTEGER(C_INT), VALUE      :: N
      TYPE(C_PTR), VALUE         :: D_X
      TYPE(C_PTR), VALUE         :: D_Y
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MLP_GRAD_DEVICE(MLP, N, D_X, D_T, LOSS) BIND(C, &
        NAME='fz_mlp_grad_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: MLP
      INTEGER(C_INT), VALUE      :: N
      TYPE(C_PTR), VALUE         :: D_X
      TYPE(C_PTR), VALUE         :: D_T
      REAL(C_FLOAT)              :: LOSS(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MLP_TRAIN_DEVICE(MLP, N, D_X, D_T, BATCH, EPOCHS, LR, SEED, LOSS) &
        BIND(C, NAME='fz_mlp_train_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: MLP
      INTEGER(C_INT), VALUE      :: N
      TYPE(C_PTR), VALUE         :: D_X
      TYPE(C_PTR), VALUE         :: D_T
      INTEGER(C_INT), VALUE      :: BATCH
      INTEGER(C_INT), VALUE      :: EPOCHS
      REAL(C_FLOAT), VALUE       :: LR
      INTEGER(C_LONG_LONG), VALUE :: SEED
      REAL(C_FLOAT)              :: LOSS(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MLP_FORWARD_OBS_DEVICE(MLP, N, D_OBS, D_MU, D_SD, D_Y, STREAM) &
        BIND(C, NAME='fz_mlp_forward_obs_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: MLP
      INTEGER(C_INT), VALUE      :: N
      TYPE(C_PTR), VALUE         :: D_OBS
      TYPE(C_PTR), VALUE         :: D_MU
      TYPE(C_PTR), VALUE         :: D_SD
      TYPE(C_PTR), VALUE         :: D_Y
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MLP_IO(MLP, NIN, NOUT) BIND(C, NAME='fz_mlp_io')
      IMPORT
      TYPE(C_PTR), VALUE         :: MLP
      INTEGER(C_INT)             :: NIN(*)
      INTEGER(C_INT)             :: NOUT(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MLP_SET_LOSS_WEIGHTS(MLP, W, N) BIND(C, &
        NAME='fz_mlp_set_loss_weights')
      IMPORT
      TYPE(C_PTR), VALUE         :: MLP
      REAL(C_FLOAT)              :: W(*)
      INTEGER(C_INT), VALUE      :: N
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_WARM_START_DEVICE(CTX, MLP, NPIX, D_OBS, D_NORM, D_BASE, &
        D_MODELS, STREAM) BIND(C, NAME='fz_warm_start_device')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      TYPE(C_PTR), VALUE         :: MLP
      INTEGER(C_INT), VALUE      :: NPIX
      TYPE(C_PTR), VALUE         :: D_OBS
      TYPE(C_PTR), VALUE         :: D_NORM
      TYPE(C_PTR), VALUE         :: D_BASE
      TYPE(C_PTR), VALUE         :: D_MODELS
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_INVERT_WARM(CTX, MLP, NORM, BASE, NPIX, OBS, TARGET_CHI2, &
        HYDROSTATIC, OPTS, MODEL_OUT, CHI2, ITERS, SYN_OUT, STATUS) BIND(C, &
        NAME='fz_invert_warm')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      TYPE(C_PTR), VALUE         :: MLP
      REAL(C_FLOAT)              :: NORM(*)
      REAL(C_FLOAT)              :: BASE(*)
      INTEGER(C_INT), VALUE      :: NPIX
      REAL(C_DOUBLE)             :: OBS(*)                 ! OBS3D(NFREQ,NPIX)
      TYPE(C_PTR), VALUE         :: TARGET_CHI2            ! per-pixel chi2 goal or C_NULL_PTR
      INTEGER(C_INT), VALUE      :: HYDROSTATIC
      TYPE(FZ_LM_OPTS)           :: OPTS
      REAL(C_FLOAT)              :: MODEL_OUT(*)           ! MODEL(NZ,13,NCOL), may be MODEL
      REAL(C_DOUBLE)             :: CHI2(*)
      INTEGER(C_INT)             :: ITERS(*)
      TYPE(C_PTR), VALUE         :: SYN_OUT                ! RSYN1D(NFREQ,NPIX) or C_NULL_PTR
      INTEGER(C_INT)             :: STATUS(*)              ! per column / pixel
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_PROFILE_ENABLE(CTX, ON) BIND(C, NAME='fz_profile_enable')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      INTEGER(C_INT), VALUE      :: ON
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_PROFILE_READ(CTX, MS, LAUNCHES, ITEMS, N) BIND(C, &
        NAME='fz_profile_read')
      IMPORT
      TYPE(C_PTR), VALUE         :: CTX
      REAL(C_DOUBLE)             :: MS(*)
      INTEGER(C_INT)             :: LAUNCHES(*)
      INTEGER(C_LONG_LONG)       :: ITEMS(*)
      INTEGER(C_INT), VALUE      :: N
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MEASURE_FP32_PEAK(DEVICE, TFLOPS) BIND(C, &
        NAME='fz_measure_fp32_peak')
      IMPORT
      INTEGER(C_INT), VALUE      :: DEVICE
      REAL(C_DOUBLE)             :: TFLOPS(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MEASURE_FP64_PEAK(DEVICE, TFLOPS) BIND(C, &
        NAME='fz_measure_fp64_peak')
      IMPORT
      INTEGER(C_INT), VALUE      :: DEVICE
      REAL(C_DOUBLE)             :: TFLOPS(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_V3_HEADER(PATH, ID, VERSION, NDIMS, DIMS) BIND(C, &
        NAME='fz_v3_header')
      IMPORT
      CHARACTER(KIND=C_CHAR)     :: PATH(*)                ! NUL-terminated
      INTEGER(C_INT)             :: ID(*)
      INTEGER(C_INT)             :: VERSION(*)
      INTEGER(C_INT)             :: NDIMS(*)
      INTEGER(C_INT), VALUE      :: DIMS
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_V3_READ_MODEL(PATH, NX, NY, NZ, CUBES) BIND(C, &
        NAME='fz_v3_read_model')
      IMPORT
      CHARACTER(KIND=C_CHAR)     :: PATH(*)                ! NUL-terminated
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      INTEGER(C_INT), VALUE      :: NZ
      REAL(C_FLOAT)              :: CUBES(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_V3_WRITE_MODEL(PATH, NX, NY, NZ, CUBES) BIND(C, &
        NAME='fz_v3_write_model')
      IMPORT
      CHARACTER(KIND=C_CHAR)     :: PATH(*)                ! NUL-terminated
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      INTEGER(C_INT), VALUE      :: NZ
      REAL(C_FLOAT)              :: CUBES(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_V3_READ_PROFILES(PATH, NX, NY, NW, IND, WAVE, STOKES) BIND(C, &
        NAME='fz_v3_read_profiles')
      IMPORT
      CHARACTER(KIND=C_CHAR)     :: PATH(*)                ! NUL-terminated
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      INTEGER(C_INT), VALUE      :: NW
      REAL(C_FLOAT)              :: IND(*)
      REAL(C_FLOAT)              :: WAVE(*)
      REAL(C_FLOAT)              :: STOKES(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_V3_WRITE_PROFILES(PATH, NX, NY, NW, IND, WAVE, STOKES) BIND(C, &
        NAME='fz_v3_write_profiles')
      IMPORT
      CHARACTER(KIND=C_CHAR)     :: PATH(*)                ! NUL-terminated
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      INTEGER(C_INT), VALUE      :: NW
      REAL(C_DOUBLE)             :: IND(*)
      REAL(C_DOUBLE)             :: WAVE(*)
      REAL(C_FLOAT)              :: STOKES(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_V3_WRITE_RFS(PATH, NX, NY, NZ, NW, Z, LOGV, IND, WAVE, DATA) &
        BIND(C, NAME='fz_v3_write_rfs')
      IMPORT
      CHARACTER(KIND=C_CHAR)     :: PATH(*)                ! NUL-terminated
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      INTEGER(C_INT), VALUE      :: NZ
      INTEGER(C_INT), VALUE      :: NW
      REAL(C_DOUBLE)             :: Z(*)
      INTEGER(C_INT)             :: LOGV(*)
      REAL(C_DOUBLE)             :: IND(*)
      REAL(C_DOUBLE)             :: WAVE(*)
      REAL(C_FLOAT)              :: DATA(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_V3_READ_RFS(PATH, NX, NY, NZ, NW, Z, LOGV, IND, WAVE, DATA) &
        BIND(C, NAME='fz_v3_read_rfs')
      IMPORT
      CHARACTER(KIND=C_CHAR)     :: PATH(*)                ! NUL-terminated
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      INTEGER(C_INT), VALUE      :: NZ
      INTEGER(C_INT), VALUE      :: NW
      REAL(C_FLOAT)              :: Z(*)
      INTEGER(C_INT)             :: LOGV(*)
      REAL(C_FLOAT)              :: IND(*)
      REAL(C_FLOAT)              :: WAVE(*)
      REAL(C_FLOAT)              :: DATA(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_V3_READ_LSF(PATH, N, YK) BIND(C, NAME='fz_v3_read_lsf')
      IMPORT
      CHARACTER(KIND=C_CHAR)     :: PATH(*)                ! NUL-terminated
      INTEGER(C_INT), VALUE      :: N
      REAL(C_DOUBLE)             :: YK(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_V3_WRITE_LSF(PATH, N, YK) BIND(C, NAME='fz_v3_write_lsf')
      IMPORT
      CHARACTER(KIND=C_CHAR)     :: PATH(*)                ! NUL-terminated
      INTEGER(C_INT), VALUE      :: N
      REAL(C_DOUBLE)             :: YK(*)
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MODEL_FROM_V3_DEVICE(NX, NY, NZ, D_CUBES, D_MODEL, STREAM) &
        BIND(C, NAME='fz_model_from_v3_device')
      IMPORT
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      INTEGER(C_INT), VALUE      :: NZ
      TYPE(C_PTR), VALUE         :: D_CUBES
      TYPE(C_PTR), VALUE         :: D_MODEL
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_MODEL_TO_V3_DEVICE(NX, NY, NZ, D_MODEL, X, Y, D_CUBES, STREAM) &
        BIND(C, NAME='fz_model_to_v3_device')
      IMPORT
      INTEGER(C_INT), VALUE      :: NX
      INTEGER(C_INT), VALUE      :: NY
      INTEGER(C_INT), VALUE      :: NZ
      TYPE(C_PTR), VALUE         :: D_MODEL
      REAL(C_DOUBLE)             :: X(*)
      REAL(C_DOUBLE)             :: Y(*)
      TYPE(C_PTR), VALUE         :: D_CUBES
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_OBS_FROM_V3_DEVICE(NPIX, NW, D_STOKES, D_OBS, STREAM) BIND(C, &
        NAME='fz_obs_from_v3_device')
      IMPORT
      INTEGER(C_INT), VALUE      :: NPIX
      INTEGER(C_INT), VALUE      :: NW
      TYPE(C_PTR), VALUE         :: D_STOKES
      TYPE(C_PTR), VALUE         :: D_OBS
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_SYN_TO_V3_DEVICE(NPIX, NW, D_SYN, D_STOKES, STREAM) BIND(C, &
        NAME='fz_syn_to_v3_device')
      IMPORT
      INTEGER(C_INT), VALUE      :: NPIX
      INTEGER(C_INT), VALUE      :: NW
      TYPE(C_PTR), VALUE         :: D_SYN
      TYPE(C_PTR), VALUE         :: D_STOKES
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
    INTEGER(C_INT) FUNCTION FZ_RF_TO_V3_DEVICE(NPIX, NZ, NW, D_RF, D_OUT, STREAM) BIND(C, &
        NAME='fz_rf_to_v3_device')
      IMPORT
      INTEGER(C_INT), VALUE      :: NPIX
      INTEGER(C_INT), VALUE      :: NZ
      INTEGER(C_INT), VALUE      :: NW
      TYPE(C_PTR), VALUE         :: D_RF
      TYPE(C_PTR), VALUE         :: D_OUT
      TYPE(C_PTR), VALUE         :: STREAM                 ! cudaStream_t or C_NULL_PTR
    END FUNCTION
  END INTERFACE
END MODULE FZ_B200
