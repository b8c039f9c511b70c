/*
 * firtez-dz B200 -- C-ABI of the GPU Stokes synthesis / pixel-wise
 * Levenberg-Marquardt path of FIRTEZ-dz.
 *
 * Plain C types only; every array is a host or device pointer plus sizes.
 * Layouts are the reference's (Fortran column-major):
 *
 *   model   MODEL(NZ,13,ncol) REAL*4, parameter order of src/atm_param.f90:38-75:
 *           1 T[K] 2 Pg[dyn cm^-2] 3 rho[g cm^-3] 4 Pe 5 mu 6 Bx[G] 7 By 8 Bz
 *           9 vx 10 vy 11 vz[cm/s] 12 log tau5 13 z[km]   (index 1 = bottom)
 *   syn     RSYN1D(NFREQ,ncol) REAL*8, NFREQ = 4*NUMW, Stokes-major blocks
 *           I(1:NUMW),Q,U,V already multiplied by GAIN (src/forward.f90:793-853)
 *   gain    GAIN1D(4,NUMW) REAL*4 (src/normalization.f90:696-754)
 *
 * Return codes: 0 = OK, < 0 = API error (fz_strerror).  Per-column status
 * words replace the reference's STOP statements.
 */
#ifndef FZ_B200_H
#define FZ_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FZ_MAXBLEND 8
#define FZ_MAXLINES 64

/* API errors */
#define FZ_ERR_ARG (-1)
#define FZ_ERR_CUDA (-2)
#define FZ_ERR_NOMEM (-3)
#define FZ_ERR_PARSE (-4)
#define FZ_ERR_LIMIT (-5)
#define FZ_ERR_STATE (-6)

/* per-column status bits */
#define FZ_OK 0
#define FZ_CHEM_NOCONV 1 /* GET_RHO: >= 100 iterations or nH < 0 (chemical_equilibrium.f90:242) */
#define FZ_NAN 2         /* non-finite opacity / Stokes (rtesolver.f90:337-352, voigt.f:88-95) */

/* One row of lines_database.dat after NREAD_LINES_DATABASE
 * (replaces the module arrays LINE_NUM, LINE_ZN, LINE_ION, LINE_L0, LOGGF,
 * EPLOW, ALPHA, SIGMA, SL..JU of src/forward_param.f90:17-21). */
typedef struct {
  int32_t num, zn, ion, flag;
  int32_t otr[2];
  int32_t abo_ierr, pad;
  double l0, loggf, eplow, alpha, sigma;
  double sl, ll, jl, su, lu, ju;
  double elowlim, eupplim;
} fz_line;

/* One spectral region of the LINES: section: IND_LINE/BLENDSID (0-based
 * indices into the line table), BLENDSDIFF [mA], NUMWAVE, WAVE_INI and
 * DELTA_LAMBDA [mA] (src/input_file.f90:290-366, src/pre_post_duties.f90:592-621). */
typedef struct {
  int32_t nblend;
  int32_t line[FZ_MAXBLEND];
  double wdif[FZ_MAXBLEND];
  int32_t numwave, pad;
  double wave_ini, dlambda;
} fz_region;

typedef struct fz_ctx fz_ctx;

/* Library version (major*100+minor). */
int fz_version(void);
const char* fz_strerror(int code);

/* Parse the text of lines_database.dat: 13- or 8-column rows terminated by
 * END, ABO collision parameters interpolated where the row leaves them 0.
 * Replaces NREAD_LINES_DATABASE (src/lines_database.f90:380-530).
 * Returns the number of rows or a negative error. */
int fz_lines_parse(const char* text, fz_line* out, int maxn);

/* Create a context on CUDA device `device` for a fixed line set and height
 * count: uploads the line table, the Zeeman patterns (ZEEMAN_COMP,
 * src/magsplit.f90:38-187, hoisted out of the z loop) and the wavelength grid
 * (WAVE_INIT).  gain may be NULL: the HSRA continuum normalisation GET_NORM
 * (src/normalization.f90:696-754) is then computed on the GPU.
 * Replaces the set-up done by START_STEP (src/pre_post_duties.f90:59-93). */
int fz_create(fz_ctx** ctx, const fz_line* lines, int nlines, const fz_region* regions, int nregions,
              int nz, const float* gain, int device);
int fz_destroy(fz_ctx* ctx);

/* Number of wavelengths NUMW of the context. */
int fz_numw(const fz_ctx* ctx);
/* Copy GAIN1D(4,NUMW) to host memory. */
int fz_get_gain(fz_ctx* ctx, float* gain);

/* hydrostatic, for the synthesis entry points (fz_forward*, not the response
 * functions or the inversion, which take 0 or 1): 0 = Pg given (GET_NHNEMU_G),
 * 1 = hydrostatic equilibrium integrated from the top (HYDRO_TOP,
 * RK4_INTEGRATION_LOG), 2 = integrated from the height of least |log tau5| of
 * the input model, Pg kept there (HYDRO_TOP off, RK4_INTEGRATION_LOG_LTAUM05,
 * src/hydrostatic_tools.f90:226-346). */
#define FZ_HE_NONE 0
#define FZ_HE_TOP 1
#define FZ_HE_LTAU 2

/* Forward synthesis of ncol columns, host buffers: the batched equivalent of
 * the worker side of FORWARD3D + FORWARD1D (src/forward.f90:106-291,
 * :857-1029) without response functions.  model is read; model_out (may be
 * NULL, may equal model) receives the updated rho, Pe, mu, log tau5 and, with
 * hydrostatic != 0, Pg (RK4_INTEGRATION_LOG, src/hydrostatic_tools.f90:150-222).
 * syn is RSYN1D(NFREQ,ncol), status is (ncol) or NULL. */
int fz_forward(fz_ctx* ctx, int ncol, const float* model, int hydrostatic, double* syn, float* model_out,
               int* status);

/* Same, with device pointers, enqueued on `stream` (a cudaStream_t, NULL =
 * default stream).  model_out is required (it may alias model).  Scratch
 * memory is owned by the context and grows on demand. */
int fz_forward_device(fz_ctx* ctx, int ncol, const float* d_model, int hydrostatic, double* d_syn,
                      float* d_model_out, int* d_status, void* stream);

/* Allocation-free variant of fz_forward_device, for callers that may not
 * allocate device memory during a call -- code running inside a host
 * framework that owns the device allocator, real-time loops, or anything
 * that has to stay free of cudaMalloc/cudaFree after start-up.  It has no
 * counterpart in the reference.  The per-call scratch (per-height nH, ne and
 * the opacity slab) lives in one file-scope 64 MiB device array instead of
 * the context's grow-on-demand buffers; the call itself calls no cudaMalloc,
 * cudaFree or allocating library routine.  Limit: ncol * nz * (16 + 4*SW)
 * bytes <= 64 MiB (SW = slab width, 20 floats for two lines; about 5400
 * columns of 128 heights); larger batches return FZ_ERR_LIMIT -- split them.
 * The array is shared by every call on a device and keeps the last call's
 * contents; every word a kernel reads is written earlier in the same call.
 * Calls that overlap on the GPU (other streams, other threads) race on it:
 * serialise them.  The first call on each device looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture.  Arguments as fz_forward_device; the context itself is created
 * (and allocated) once by fz_create. */
int fz_forward_device_static(fz_ctx* ctx, int ncol, const float* d_model, int hydrostatic, double* d_syn,
                             float* d_model_out, int* d_status, void* stream);

/* The model-only modes of FIRTEZ-dz (MODE h / t, src/invert3d.f90:159-178):
 *   fz_hydrostatic: hydrostatic equilibrium only (MGETHEQ; FORWARD1D stops
 *     after the HE integration, src/forward.f90:890-909): Pg, rho, Pe, mu of
 *     model_out; hydrostatic = FZ_HE_TOP or FZ_HE_LTAU.
 *   fz_log_tau5: the GETTAU mode (MGETTAU): chemistry (HE as hydrostatic
 *     says), the continuum opacity at 5000 A and log tau5 from the top
 *     (src/forward.f90:1000-1006), without the Stokes synthesis.
 * model_out may equal model; status as fz_forward. */
int fz_hydrostatic(fz_ctx* ctx, int ncol, const float* model, int hydrostatic, float* model_out, int* status);
int fz_hydrostatic_device(fz_ctx* ctx, int ncol, const float* d_model, int hydrostatic, float* d_model_out,
                          int* d_status, void* stream);
int fz_log_tau5(fz_ctx* ctx, int ncol, const float* model, int hydrostatic, float* model_out, int* status);
int fz_log_tau5_device(fz_ctx* ctx, int ncol, const float* d_model, int hydrostatic, float* d_model_out,
                       int* d_status, void* stream);

/* Response functions.  fz_rf_nodes selects the free parameters and their
 * node counts, nodes[p-1] for the reference parameter p of atm_param.f90
 * (1 T, 2 Pg, 4 Bx, 5 By, 6 Bz, 7 v_z; 3 rho and 8 P0 must be 0); the hat
 * interpolation of GET_INT_COEFS (src/get_dmodel.f90:563-644) maps nodes to
 * heights, so nodes[p-1] == nz gives the response at every height.  Returns
 * NP = sum of the node counts (<= 1024) or a negative error.  Layouts whose
 * node accumulators fit in shared memory (4 NP floats per wavelength) are
 * accumulated along z in the RF kernel; larger ones (e.g. every height of T
 * and v_z, the reference's last cycle) are contracted from the response
 * functions at every height.  Replaces the node set-up of UPDATE_COEFS
 * (src/get_dmodel.f90:648-721). */
int fz_rf_nodes(fz_ctx* ctx, const int* nodes /* [8] */);

/* Forward synthesis with response functions: as fz_forward plus the node
 * Jacobian EQVDSYN(NFREQ, NP) of every column, REAL*4, Stokes-major rows
 * (I,Q,U,V blocks of NUMW) x GAIN, parameters in reference order with their
 * nodes -- FORWARD1D with MRESPFUNCT followed by OLD_DSYN_PROPAGATION and
 * CALCULATE_EQUIVALENT_DSYN (src/forward.f90:511-681, :857-1029).  jac is
 * (NFREQ, NP, ncol).  With hydrostatic != 0 the T response carries the
 * reference's global term through the pressure stratification and the B and
 * v_z responses use the layer's outgoing Stokes vector, as the reference's
 * OLD_ANALYTICAL_SOLVER does (src/rtesolver.f90:218-260).  FZ_ERR_STATE if
 * fz_rf_nodes was not called. */
int fz_forward_rf(fz_ctx* ctx, int ncol, const float* model, int hydrostatic, double* syn, float* jac,
                  float* model_out, int* status);
int fz_forward_rf_device(fz_ctx* ctx, int ncol, const float* d_model, int hydrostatic, double* d_syn,
                         float* d_jac, float* d_model_out, int* d_status, void* stream);

/* Forward synthesis with the response functions at every height, the
 * WRITE RESPONSE FUNCTION output (src/pre_post_duties.f90:331-353): the
 * EQVDSYN of CALCULATE_EQUIVALENT_DSYN with NJ = NZ for each of T, Pg, Bx,
 * By, Bz, v_z (src/forward.f90:552-681), i.e. rf is (NFREQ, 6 NZ, ncol)
 * REAL*4, parameter blocks of NZ heights in that order, x GAIN; the same
 * hydrostatic conventions as fz_forward_rf.  Needs no fz_rf_nodes call.
 * 2.75 MB of rf per column at NZ = 128, NUMW = 224 (plus a device scratch of
 * the per-layer operators, 64 B per height and wavelength): callers stream
 * large fields in batches. */
int fz_forward_rf_full(fz_ctx* ctx, int ncol, const float* model, int hydrostatic, double* syn, float* rf,
                       float* model_out, int* status);
int fz_forward_rf_full_device(fz_ctx* ctx, int ncol, const float* d_model, int hydrostatic, double* d_syn,
                              float* d_rf, float* d_model_out, int* d_status, void* stream);

/* Launch-shape autotuner (no counterpart in the reference).  The shapes
 * live in the context and apply to every later call on it:
 *   chain_warps            warps per block of the chemistry chain kernel,
 *                          1..4
 *   chain_lanes            lanes per column of the chemistry chain kernel:
 *                          32 (one column per warp), 16 (two), or 0 (16
 *                          for batches of at least 16 columns per SM, else
 *                          32; the default)
 *   chemder_blocks_per_sm  grid cap of the chemistry-derivative kernel per
 *                          SM (0 = one block per 4 heights)
 *   opac_rf_threads        block size of the opacity-derivative kernel
 *                          (64, 128 or 256)
 *   lm_slots               pixels in flight of the inversion when
 *                          fz_lm_opts.slots is 0
 * fz_autotune_forward times the candidates of the first three on ncol
 * device columns; fz_autotune_lm inverts the same npix pixels once per
 * candidate slot count and keeps the highest pixels/s.  The *_ms and
 * lm_pixels_per_s fields report the winners' timings. */
typedef struct {
  int chain_warps, chemder_blocks_per_sm, opac_rf_threads, lm_slots;
  float chain_ms, chemder_ms, opac_rf_ms, lm_pixels_per_s;
  int chain_lanes, pad;
} fz_tune;
int fz_autotune_forward(fz_ctx* ctx, int ncol, const float* d_model, int hydrostatic, fz_tune* out);
int fz_tune_get(fz_ctx* ctx, fz_tune* out);
int fz_tune_set(fz_ctx* ctx, const fz_tune* t);

/* SMOOTHING_B (src/model_spatial_extension.f90:351-491), which
 * INITIALIZE_CYCLE applies to the models of the free parameters at the start
 * of every cycle, the first included (src/invert3d.f90:228-325): a 1-2-1
 * average in FP64 along x, then y, then height, the end points of each
 * direction kept and directions of 4 or fewer points left alone, rounded to
 * REAL*4.  models: MODEL(NZ,13,NY*NX) with pixel iy + NY*ix (the order of
 * the reference's (NZ,NY,NX) cubes), smoothed in place.  params[8] flags the
 * reference parameters to smooth (1..8 = T, Pg, rho, Bx, By, Bz, v_z, P0; P0
 * smooths Pg); NULL: the free parameters of fz_rf_nodes. */
int fz_smooth(fz_ctx* ctx, int nx, int ny, float* models, const int* params);
int fz_smooth_device(fz_ctx* ctx, int nx, int ny, float* d_models, const int* params, void* stream);

/* Options of the batched inversion (the reference's control-file values in
 * brackets): maxsteps, the per-pixel limit on the STEPS counter of
 * UPDATE_LAMBDA (MAXITER, 5); maxit, a hard cap on iterations per pixel;
 * dchi2, an accepted step whose relative chi2 gain is below it ends the
 * pixel (0 = off); svdtol, the relative SVD cut (RSVDTOL, 1e-4); isigma, the
 * noise (NOISE, 4e-3); wstk, the Stokes weights (1,1,1,1); slots, the number
 * of pixels in flight (0 = the tuned count, 8192 untuned).  fallback and
 * fallback_model (no counterpart in the reference): with a per-pixel chi2
 * goal, a pixel whose search ends above fallback x its goal starts once more
 * from fallback_model (device, one MODEL(NZ,13) for every pixel, e.g. the
 * default guess) in the same slot pool, keeping the goal; its iterations
 * add up.  0 / NULL: off.  fallback_model is a device pointer for
 * fz_invert_device and a host pointer for fz_invert.  reg_type, reg_alpha:
 * the vertical regularisation of VERTICAL REGULARIZATION
 * (GET_IT_PENALTIES, src/get_dmodel.f90:1041-1197), per reference parameter
 * 1..8: type 0 (node values to zero, D = diag(1/NJ)) or 1 (differences to
 * the previous node) and PEN_ALP (0: off); chi2 gains sum(PEN_RES^2) of the
 * current model, the normal equations PEN_HSS and -PEN_RES of the best.
 * fallback_steps: with fallback on, a pixel restarts as soon as its
 * stagnation counter (the STEPS of UPDATE_LAMBDA) reaches fallback_steps
 * while its best chi2 is still above fallback x its goal, instead of when
 * its search ends (0: when it ends; negative: at its first evaluation, i.e.
 * the initial model itself decides).  fallback_free: 1 = the restarted
 * search ignores the goal and runs to the plain stop rules, 0 = it keeps
 * the goal.
 * solver: SOLVER_METHOD (MISC SETUP LINEAR_SOLVER), 1 (or 0) = the SVD
 * pseudo-inverse of GET_INVERSE, 2 = the conjugate-gradient iteration of
 * NEW_CALCULATE_DELTA_UBICGSTAB (src/lm.f90:375-453).  node_expansion:
 * NODE_EXPANSION (PERTURBATION_TYPE), 1 (or 0) = SIR/NICOLE-like node
 * perturbations, 2 = STiC-like (the expanded node values are the new
 * profile; src/get_dmodel.f90:1792-1804).
 * assist: SET_TAU's initial-guess assists for fz_invert_cycles_device
 * (FZ_ASSIST_* bits; the control file's ASSIST line and PROGRESSIVE).
 * global_stop: MAKE_DECISION's field-wide rule (src/invert3d.f90:843-846):
 * every pixel of the call stops once the mean of STEPS over its npix pixels
 * reaches max(1, maxsteps - cycles_left), cycles_left being MAXITER - CURIC
 * (0 in the last or only cycle; fz_invert_cycles_device sets it per cycle).
 * The rule is defined for a field iterating in lockstep, so with it on all
 * pixels are in flight at once (slots = npix).  state_out: (5, npix) REAL*8,
 * the final INV_SLA(1:4) and INV_SLA(9) of each pixel -- STEPS, chi2 of its
 * last model, best chi2, PRECYC, lambda (src/invert3d.f90:275-286) --; a
 * device pointer for fz_invert_device, a host pointer for fz_invert; NULL:
 * not written. */
#define FZ_ASSIST_TEMP 1
#define FZ_ASSIST_PGAS 2
#define FZ_ASSIST_BVEC 4
#define FZ_ASSIST_VLOS 8
#define FZ_ASSIST_PROGRESSIVE 16
typedef struct {
  int maxsteps, maxit;
  double dchi2, svdtol, isigma;
  float wstk[4];
  int slots, assist;
  double fallback;
  const float* fallback_model;
  int reg_type[8];
  double reg_alpha[8];
  int fallback_steps, solver, node_expansion, global_stop;
  int cycles_left, fallback_free;
  double* state_out;
} fz_lm_opts;

/* Batched pixel-wise Levenberg-Marquardt inversion of npix pixels with the
 * node layout of fz_rf_nodes: the cycle loop of INVERT3D
 * (src/invert3d.f90:57-178) with GET_DMODEL3DS/GET_PERT_1D per pixel
 * (src/get_dmodel.f90:1201-1577), each pixel iterating until its own stop
 * rule, finished pixels replaced from a device work queue.  obs is
 * OBS3D(NFREQ, npix) (Stokes-major, GAIN-normalised, as RSYN1D); init is the
 * initial model MODEL(NZ,13,npix).  Outputs: the best model, its chi2
 * (NEW_CALCULATE_CHI2 normalisation), the iterations used, optionally the
 * best synthesis (syn_out, may be NULL) and a status per pixel.  Layouts
 * of up to 16 nodes solve with one warp per pixel (mma.sync normal
 * equations, warp Jacobi SVD / CG); up to 1024 nodes with the tcgen05
 * normal equations and a CTA per pixel for the FP64 SVD or CG, the slot
 * count then held within a 24 GB working set. */
int fz_invert(fz_ctx* ctx, int npix, const double* obs, const float* init, const double* target_chi2,
              int hydrostatic, const fz_lm_opts* opts, float* model_out, double* chi2, int* iters,
              double* syn_out, int* status);
/* Device-pointer variant.  In both, target_chi2 (npix, may be NULL) adds a
 * per-pixel goal: a pixel also stops once its best chi2 is at or below its
 * goal (e.g. the chi2 another start reached on the same pixel). */
int fz_invert_device(fz_ctx* ctx, int npix, const double* d_obs, const float* d_init,
                     const double* d_target_chi2, int hydrostatic, const fz_lm_opts* opts,
                     float* d_model_out, double* d_chi2, int* d_iters, double* d_syn_out, int* d_status,
                     void* stream);

int fz_autotune_lm(fz_ctx* ctx, int npix, const double* d_obs, const float* d_init, const double* d_target_chi2,
                   int hydrostatic, const fz_lm_opts* opts, const int* candidates, int ncand, fz_tune* out);

/* SMOOTHING_B of one shard of a field split over ranks by x: the shard's
 * nx columns are field columns x0 .. x0+nx-1 of an nx_field-column field
 * (pixel iy + NY*ix within the array).  The array may carry the neighbours'
 * halo columns at its ends (then x0 and nx count them): the x pass reads
 * them, the field's own first and last columns are kept and its 4-point
 * rule applies, so the interior columns come out as in the whole field's
 * SMOOTHING_B.  fz_smooth_device is the whole-field case (x0 = 0,
 * nx_field = nx). */
int fz_smooth_shard_device(fz_ctx* ctx, int nx, int ny, int x0, int nx_field, float* d_models, const int* params,
                           void* stream);

/* INVERT3D's cycle loop (src/invert3d.f90:57-178, :228-408) on device
 * buffers for an NX x NY field (pixel iy + NY*ix): for each cycle the node
 * layout nodes[8*cycle .. 8*cycle+7] (fz_rf_nodes), SMOOTHING_B of the
 * current models (fz_smooth_device), the batched inversion from them with a
 * fresh LM state per pixel (fz_invert_device), then END_CYCLE's plain
 * synthesis of the best models, which become the next cycle's models.
 * d_models (MODEL(NZ,13,NX*NY)) holds the initial models on entry and the
 * final ones on return; d_chi2, d_iters, d_status are those of the last
 * cycle.  The context keeps the last cycle's node layout. */
int fz_invert_cycles_device(fz_ctx* ctx, int nx, int ny, const double* d_obs, float* d_models, int ncycles,
                            const int* nodes, int hydrostatic, const fz_lm_opts* opts, double* d_chi2, int* d_iters,
                            int* d_status, void* stream);

/* Line spread function of a spectral region (LSF_INIT, src/pre_post_duties.f90:
 * 742-900; applied by CALCULATE_EQUIVALENT_SYN1D / _DSYN, src/forward.f90:
 * 615-657, :793-853): every synthesis row and every node-Jacobian (and full
 * response-function) row of the region is circularly convolved with the
 * region's kernel YK, in FP64, the result rounded to REAL*4.
 *   fz_lsf_gaussian: the reference's Gaussian of sigma and centre w0 [mA]
 *     over the region's NUMWAVE points (step WAVE(WI+1) - WAVE(WI)).
 *   fz_lsf_kernel:   a kernel as READ_LSF_FILE gives it (n = NUMWAVE of the
 *     region, index 0 = the centre, as the reference convolves it).
 * A kernel is valid when its sum is within 0.01 of 1 (then renormalised);
 * both return 1 (valid, the region is convolved from now on) or 0 (the
 * region is left unconvolved, as the reference does).  fz_lsf_clear turns
 * the LSF off.  Applies to every later synthesis, RF and inversion call. */
int fz_lsf_gaussian(fz_ctx* ctx, int region, double sigma, double w0);
int fz_lsf_kernel(fz_ctx* ctx, int region, const double* yk, int n);
int fz_lsf_clear(fz_ctx* ctx);

/* SET_TAU's assists (src/invert3d.f90:492-727) on an NX x NY field (pixel
 * iy + NY*ix) before a cycle: from the observations' Stokes I of the first
 * spectral region summed over the field, three template vectors (the
 * normalised sum and its two centred derivatives); per pixel, with field
 * maxima as the scale:
 *   FZ_ASSIST_BVEC  Bx, By from the Q, U projections on the second
 *                   derivative (azimuth atan2(U,Q)/2, 1000 G at the field
 *                   maximum), Bz from the V projection on the first (-1000 G)
 *   FZ_ASSIST_VLOS  v_z from the I projection on the first derivative less
 *                   its component along the sum (-2 km/s at the maximum)
 *   FZ_ASSIST_TEMP  T shifted so that T at height CEILING(NZ/3) is the
 *                   brightness temperature of the mean I (6390 K at I = 1)
 *   FZ_ASSIST_PGAS  Pg scaled to 1.333e5 at that height
 * with TEMP or PGAS, a plain synthesis then updates rho, Pe, mu and log tau5:
 * hydrostatic != 0 integrates Pg from the anchor log tau5 = 0 the assists
 * set (hydrostatic mode 2 of fz_forward), else Pg is kept.  Constant-in-
 * height B and v_z, as the reference. */
int fz_set_tau_device(fz_ctx* ctx, int nx, int ny, const double* d_obs, float* d_models, int assist, int hydrostatic,
                      void* stream);
int fz_set_tau(fz_ctx* ctx, int nx, int ny, const double* obs, float* models, int assist, int hydrostatic);

/* SET_TAU on one shard of a field split over ranks by x (contiguous runs of
 * columns, pixel iy + NY*ix within the shard): the per-pixel work as
 * fz_set_tau_device, its two field-wide reductions through the caller's
 * reduce(user, kind, data, n, nx), which returns 0 on success:
 *   kind 0: data (nx * n doubles, x-major) holds this shard's sums of Stokes
 *           I over y per column (n = NUMWAVE of the first region); it must
 *           leave in data[0 .. n) the field total, every shard's columns
 *           summed in field x order (the reference's SUM order);
 *   kind 1: data (3) holds this shard's maxima of the three projections;
 *           it must leave the field maxima.
 * Every shard then computes the same template vectors and scales, so the
 * result equals the whole field's.  With reduce NULL: fz_set_tau_device. */
typedef int (*fz_field_reduce_fn)(void* user, int kind, double* data, int n, int nx);
int fz_set_tau_shard_device(fz_ctx* ctx, int nx, int ny, const double* d_obs, float* d_models, int assist,
                            int hydrostatic, fz_field_reduce_fn reduce, void* user, void* stream);

/* The errors mode (GET_ERRORS3DS / GET_ERROR_1D / NEW_SOLVE_ERRORS,
 * src/get_dmodel.f90:1248-1323, :1581-1703), replacing the per-pixel worker
 * loop: for the models (usually the inversion's best), with the node layout
 * of fz_rf_nodes, the synthesis and node Jacobian, chi2 (as
 * NEW_CALCULATE_CHI2; the penalties of opts->reg_* included), per node
 * sigma_i = sqrt((chi2 / NFREQ) / H_ii) with H = Jn^T Jn the normalised
 * Jacobian's Gram diagonal, mapped to heights by REARANGE_DA_MODEL's errors
 * branch (limits [0, 1e20], node values clipped at 0.15 PARAM_NORM).
 * err: MODEL(NZ,13,npix), the rows of parameters without nodes zero (the
 * E*3D cubes of ESPLIT_MODEL3D); chi2 (npix); status may be NULL.  opts
 * supplies isigma, wstk and reg_*; the LM fields are unused.  Node layouts
 * of up to 16 nodes (FZ_ERR_LIMIT above). */
int fz_errors_device(fz_ctx* ctx, int npix, const double* d_obs, const float* d_models, int hydrostatic,
                     const fz_lm_opts* opts, float* d_err, double* d_chi2, int* d_status, void* stream);
int fz_errors(fz_ctx* ctx, int npix, const double* obs, const float* models, int hydrostatic, const fz_lm_opts* opts,
              float* err, double* chi2, int* status);

/* Batched GET_PERTURBATION (src/lm.f90:137-204) on host buffers, the call
 * at src/get_dmodel.f90:799-803: for each pixel H = J^T J (tensor cores,
 * split-bf16 x3 of the FP32-rounded Jacobian, FP32 accumulation), g = J^T
 * diff, then with dtype 1 (0 taken as 1) (H + lambda diag H)^+ g by an FP64
 * Jacobi SVD with singular values below svdtol * max dropped (GET_INVERSE,
 * :61-133; svdtol <= 0: RSVDTOL 1e-4), with dtype 2 the conjugate-gradient
 * solve (NEW_CALCULATE_DELTA_UBICGSTAB, :375-453).  jac is IJACOBIAN(NF,NP)
 * REAL*8 per pixel, (nfreq, np, npix); diff (nfreq, npix); lambda (npix);
 * reg_pen (np, npix) and reg_hss (np, np, npix), may be NULL: REG_PEN is
 * subtracted from J^T diff and REG_HSS added to J^T J as the reference does
 * (:169-174); delta (np, npix), NaN entries zeroed (NEW_SOLVE_PERTURBATION).
 * np <= 1024 (above 16: tcgen05 normal equations, CTA-wide FP64 solvers),
 * nfreq a multiple of 4. */
int fz_lm_perturbation(fz_ctx* ctx, int npix, int np, int nfreq, const double* jac, const double* diff,
                       const double* lambda, const double* reg_pen, const double* reg_hss, int dtype, double svdtol,
                       double* delta);
/* The same with the Jacobian as REAL*4 (nfreq, np, npix), e.g. the
 * normalised EQVDSYN the library itself produces (no counterpart routine:
 * the reference widens EQVDSYN to REAL*8 before GET_PERTURBATION). */
int fz_lm_perturbation_f32(fz_ctx* ctx, int npix, int np, int nfreq, const float* jac, const double* diff,
                           const double* lambda, const double* reg_pen, const double* reg_hss, int dtype,
                           double svdtol, double* delta);

/* Batched UPDATE_LAMBDA (src/get_dmodel.f90:917-956, FACTOR = 0.01) of n
 * pixels, the per-iteration lambda rule of GET_PERT_1D: chicur is the chi2
 * of the model just synthesised (1e300 for a failed synthesis); chipre
 * (best chi2), lambda, steps (STEPS) and precyc (PRECYC) are updated in
 * place -- an improvement sets chipre = chicur and divides lambda by
 * sqrt(10), lowering steps by one when it gains more than 1 % of chipre and
 * raising it otherwise; no improvement multiplies lambda by 3 when precyc is
 * 1 (which it clears) or else by 10, and raises steps; lambda >= 1e-2.  The
 * batched inversion applies the same rule in its accept step.  Host arrays,
 * or device arrays with the _device variant (enqueued on stream). */
int fz_lm_update_lambda(int n, const double* chicur, double* chipre, double* lambda, double* steps, double* precyc);
int fz_lm_update_lambda_device(int n, const double* d_chicur, double* d_chipre, double* d_lambda, double* d_steps,
                               double* d_precyc, void* stream);

/* Batched LIMIT_PERTURBATION -> REARANGE_DA_MODEL (src/get_dmodel.f90:
 * 884-907, :1843-2016) with SORT_DELTA_TO_ATMOSPHERE (:1715-1836): the node
 * perturbation delta (np, npix), normalised by PARAM_NORMS, applied to
 * MODEL(NZ,13,npix) in place with the node layout of fz_rf_nodes -- node
 * deltas clipped at 0.15 max(|node average|, PARAM_NORM), node_expansion 1
 * (or 0; SIR-like: CONTRACT(EXPAND(avg + delta) - profile) expanded again)
 * or 2 (STiC-like: the expanded clipped node values are the new profile),
 * LOWLIM/UPPLIM, and the log tau5 taper of T (:1975-1989).  The batched
 * inversion applies the same update to every trial model. */
int fz_lm_rearange(fz_ctx* ctx, int npix, float* models, const double* delta, int node_expansion);
int fz_lm_rearange_device(fz_ctx* ctx, int npix, float* d_models, const double* d_delta, int node_expansion,
                          void* stream);

/* The formal solution on given absorption matrices: SET_BOUNDARY +
 * OLD_ANALYTICAL_SOLVER with EVOL_OPERATOR (src/rtesolver.f90:163-473,
 * :1134-1147; the per-(K, lambda) calls at src/forward.f90:971-975), for a
 * host that builds its own absorption matrix.  From the bottom up, I =
 * (S, 0, 0, 0) at the first height and wherever bnd is set, else I_K =
 * (1 - O_K) S_K + O_K I_{K-1} with O_K the evolution operator of the height's
 * matrix over dz = 1e5 |z_{K+1} - z_K| cm (the top height: its backward
 * difference).  eta: (NW, 7, NZ, ncol) REAL*4, per height the seven arrays
 * ETAI, ETAQ, ETAU, ETAV, RHOQ, RHOU, RHOV in cm^-1; src: (NW, NZ, ncol)
 * source function; zz: ZZ(NZ) in km; bnd: (NZ, ncol) boundary flags or NULL;
 * out: SYN1D(4, NW, ncol) REAL*8 (without GAIN).  FP32 arithmetic, as in the
 * synthesis kernels. */
int fz_rte_solve(int ncol, int nz, int nw, const float* eta, const float* src, const double* zz, const int* bnd,
                 double* out);
int fz_rte_solve_device(int ncol, int nz, int nw, const float* d_eta, const float* d_src, const double* d_zz,
                        const int* d_bnd, double* d_out, void* stream);

/* VOIGT (src/voigt.f:17-98) on arrays, in the FP32 form the synthesis
 * kernels evaluate: H(a, v) and the Faraday-Voigt F(a, v) (the reference's
 * HH, FF) of n (damping, v) pairs, host buffers. */
int fz_voigt(int n, const float* a, const float* v, float* h, float* f);

/* Warm-start network (no counterpart in the reference): an MLP of nlayers
 * fully connected layers dims[0] -> dims[1] -> ... -> dims[nlayers] with GELU
 * between layers, trained and evaluated with hand-written BF16 tcgen05
 * tensor-core kernels (FP32 accumulation in tensor memory, FP32 master
 * weights, Adam).  dims[0..nlayers-1]
 * must be multiples of 8.  Weights start from a seeded uniform
 * Glorot initialisation.  Parameters are exchanged as FP32 in layer order
 * (W0[out][in], b0, W1, b1, ...); fz_mlp_get_params with grads != 0 returns
 * the gradients of the last fz_mlp_grad_device call instead.  Rows are
 * row-major FP32 on the device; the loss is the mean squared error. */
typedef struct fz_mlp fz_mlp;
int fz_mlp_create(fz_mlp** mlp, int nlayers, const int* dims, unsigned long long seed, int device);
int fz_mlp_destroy(fz_mlp* mlp);
long long fz_mlp_nparams(const fz_mlp* mlp);
int fz_mlp_get_params(fz_mlp* mlp, float* host, int grads);
int fz_mlp_set_params(fz_mlp* mlp, const float* host);
int fz_mlp_forward_device(fz_mlp* mlp, int n, const float* d_x, float* d_y, void* stream);
int fz_mlp_grad_device(fz_mlp* mlp, int n, const float* d_x, const float* d_t, float* loss);
int fz_mlp_train_device(fz_mlp* mlp, int n, const float* d_x, const float* d_t, int batch, int epochs, float lr,
                        unsigned long long seed, float* loss);
/* Forward of observed Stokes rows: d_obs (n x dims[0]) FP64, standardised
 * with d_mu and d_sd (dims[0] each, FP32) as they are converted to the bf16
 * inputs; d_y (n x dims[nlayers]) FP32.  Ordered after the work on stream,
 * which waits for it.  fz_mlp_io: the input and output widths. */
int fz_mlp_forward_obs_device(fz_mlp* mlp, int n, const double* d_obs, const float* d_mu, const float* d_sd,
                              float* d_y, void* stream);
int fz_mlp_io(const fz_mlp* mlp, int* nin, int* nout);
/* Per-output weights of the training loss, sum_j w_j (y_j - t_j)^2 / (n nout)
 * (host array of dims[nlayers] finite values >= 0; w NULL restores equal
 * weights).  The warm start weights each node by the chi2 its error costs
 * to first order, so that the loss approximates the chi2 of the prior. */
int fz_mlp_set_loss_weights(fz_mlp* mlp, const float* w, int n);

/* The learned initial guess of the inversion (no counterpart in the
 * reference, whose LM starts from the control file's model or SET_TAU's
 * assists): the network maps each pixel's observed Stokes vector OBS3D(NFREQ)
 * to the node values of the context's layout (fz_rf_nodes; outputs in node
 * order, standardised), and each free parameter's row of the base model
 * MODEL(NZ,13) moves by EXPAND(nodes - CONTRACT(base)) -- the way the
 * inversion perturbs a model (src/get_dmodel.f90:839-880); the other rows
 * are the base model's.  norm: FP32 x mean (NFREQ), x spread (NFREQ), node
 * mean (NP), node spread (NP).  fz_warm_start_device: device buffers,
 * models MODEL(NZ,13,npix), enqueued on stream.  fz_invert_warm: host
 * buffers -- the observations cross to the device once, the warm-start
 * models are built there and inverted by fz_invert's batched LM (other
 * arguments as fz_invert). */
int fz_warm_start_device(fz_ctx* ctx, fz_mlp* mlp, int npix, const double* d_obs, const float* d_norm,
                         const float* d_base, float* d_models, void* stream);
int fz_invert_warm(fz_ctx* ctx, fz_mlp* mlp, const float* norm, const float* base, int npix, const double* obs,
                   const double* target_chi2, int hydrostatic, const fz_lm_opts* opts, float* model_out,
                   double* chi2, int* iters, double* syn_out, int* status);

/* Per-kernel timing: when enabled, every launch of the context is bracketed
 * by CUDA events on its stream; fz_profile_read returns the accumulated
 * milliseconds, launch counts and processed columns (or LM slots; items
 * may be NULL) of the kernels (names in order:
 * "k_chain", "k_opac", "k_synth", "k_opac_rf", "k_synth_rf", "k_lm_fill",
 * "k_lm_accept", "k_lm_normal", "k_lm_solve", "k_lm_update", "k_chemder", "k_rf_prop", "k_lsf",
 * "k_saha", "k_chain_pre": the chain of a batch of at most 1024 columns on
 * k_saha's precomputed Saha factors) and resets
 * them; returns the kernel count.  Replaces the reference's
 * SYSTEM_CLOCK "Forward 3D:" timer (src/forward.f90:99-100, :295-297). */
int fz_profile_enable(fz_ctx* ctx, int on);
int fz_profile_read(fz_ctx* ctx, double* ms, int* launches, long long* items, int n);

/* Peak FP32 FMA throughput of device `device` in TFLOP/s (2 FLOP per FMA),
 * measured by a register-resident FMA-chain kernel; the denominator of the
 * FP32-pipe roofline of the synthesis kernel. */
int fz_measure_fp32_peak(int device, double* tflops);
/* The FP64 FMA peak of the device (independent FMA chains), TFLOP/s. */
int fz_measure_fp64_peak(int device, double* tflops);

/* ---------------------------------------------------------------- v3 files
 * The model, profile and response-function files of src/misc.f90, as the
 * Fortran host reads and writes them (READ_MODEL / READ_MODEL_3D :78-553,
 * WRITE_MODEL3D_V3 :801-929, READ_PROFILE_3D :1338-1642,
 * WRITE_PROFILES3D_V3 :1147-1249, WRITE_RFS3D_V3 :1862-1999): Fortran
 * unformatted sequential records, REAL*4 payloads, a header record
 * (3000+v, 3000-v, ID, NRECS, NDIMS, dims...), data records of at most
 * 268,435,446 values.  Host functions (no GPU); the payload is moved as it
 * lies in the file:
 *   model cubes   (NZ,NY,NX) x 13 in file order: T, Pg, rho, Bx, By, Bz, vz,
 *                 Pe, mu, log tau5, x, y, z
 *   profiles      STOKES(4,NW,NY,NX)
 *   RFs           DSTOKES(P,4,NW,NZ,NY,NX), P over the LOGV-flagged of
 *                 T, Pg, rho, Bx, By, Bz, vz, P0
 * The layout changes to MODEL(NZ,13,npix), OBS3D(NFREQ,npix) and the RF
 * output of fz_forward_rf_full are the fz_*_v3_device kernels below.
 * Errors: FZ_ERR_ARG (open/write failure, bad argument), FZ_ERR_PARSE (not
 * such a file, or truncated), FZ_ERR_LIMIT (dimensions differ from the
 * caller's). */
int fz_v3_header(const char* path, int* id, int* version, int* ndims, int dims[8]);
int fz_v3_read_model(const char* path, int nx, int ny, int nz, float* cubes);
int fz_v3_write_model(const char* path, int nx, int ny, int nz, const float* cubes);
int fz_v3_read_profiles(const char* path, int nx, int ny, int nw, float* ind /* NULL ok */, float* wave /* NULL ok */,
                        float* stokes);
int fz_v3_write_profiles(const char* path, int nx, int ny, int nw, const double* ind, const double* wave,
                         const float* stokes);
/* logv[8]: 1 for each of T, Pg, rho, Bx, By, Bz, vz, P0 present in data */
int fz_v3_write_rfs(const char* path, int nx, int ny, int nz, int nw, const double* z, const int* logv,
                    const double* ind, const double* wave, const float* data);
/* Returns the number of parameters present (>= 0); with data NULL only the
 * small records are read (call again with a buffer of that many
 * parameters). */
int fz_v3_read_rfs(const char* path, int nx, int ny, int nz, int nw, float* z, int* logv, float* ind, float* wave,
                   float* data);

/* Line spread function files (READ_LSF_FILE, misc.f90:2422-2555; the
 * reference's Python write_lsf): header 3003, 2997, 3330904, NRECS+1, 1, NW,
 * then NW REAL*4 values. */
int fz_v3_read_lsf(const char* path, int n, double* yk);
int fz_v3_write_lsf(const char* path, int n, const double* yk);

/* Layout changes on the device (stream-ordered, no allocation except the
 * x/y vectors of fz_model_to_v3_device):
 *   fz_model_from_v3_device  cubes -> MODEL(NZ,13,NY*NX): T, Pg, rho, Pe, mu,
 *       Bx, By, Bz, vx = vy = 0, vz, log tau5, and z = the first pixel's z
 *       column for every pixel (JOIN_MODEL2, src/forward.f90:363-405, with
 *       ZZ from READ_MODEL_3D's Z(:) = TMP(:,1,1))
 *   fz_model_to_v3_device    MODEL -> cubes, x and y cubes REAL(X(ix)),
 *       REAL(Y(iy)) from host vectors, z cube from each pixel's z row
 *       (WRITE_MODEL3D_V3)
 *   fz_obs_from_v3_device    STOKES(4,NW,NY,NX) REAL*4 -> OBS3D(4*NW,npix)
 *       REAL*8, Stokes-major blocks (ALLOCATE_AND_READ, src/pre_post_duties.f90:421-431)
 *   fz_syn_to_v3_device      RSYN1D(4*NW,npix) REAL*8 -> STOKES REAL*4
 *       (WRITE_STOKES_PROFILES, src/pre_post_duties.f90:235-245)
 *   fz_rf_to_v3_device       fz_forward_rf_full's (4*NW,NZ,6,npix) -> the
 *       DSTOKES payload with LOGV = T, Pg, Bx, By, Bz, vz
 *       (WRITE_RESPONSE_FUNCTIONS, src/pre_post_duties.f90:316-356) */
int fz_model_from_v3_device(int nx, int ny, int nz, const float* d_cubes, float* d_model, void* stream);
int fz_model_to_v3_device(int nx, int ny, int nz, const float* d_model, const double* x, const double* y,
                          float* d_cubes, void* stream);
int fz_obs_from_v3_device(int npix, int nw, const float* d_stokes, double* d_obs, void* stream);
int fz_syn_to_v3_device(int npix, int nw, const double* d_syn, float* d_stokes, void* stream);
int fz_rf_to_v3_device(int npix, int nz, int nw, const float* d_rf, float* d_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FZ_B200_H */
