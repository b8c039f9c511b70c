/*
 * TEST INFRASTRUCTURE -- not part of the product.
 *
 * FP64 CPU restatement ("oracle") of the FIRTEZ-dz hot path, used only by
 * tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py as the
 * checker.  Every routine cites the reference file:line it follows.
 *
 * Layouts follow the reference (Fortran column-major):
 *   model  : MODEL(NZ,13) REAL*4 per column, parameters in the order of
 *            src/atm_param.f90:38-75  (T, Pg, rho, Pe, mu, Bx, By, Bz, vx, vy,
 *            vz, log tau5, z[km])
 *   stokes : RSYN1D(4*NUMW) REAL*8, Stokes-major blocks of NUMW
 *            (src/forward.f90:793-853)
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One row of lines_database.dat after NREAD_LINES_DATABASE
 * (src/lines_database.f90:380-530). */
typedef struct {
  int32_t num;      /* column 1: database id                     */
  int32_t zn;       /* atomic number                              */
  int32_t ion;      /* ionisation stage (1 = neutral)             */
  int32_t flag;     /* OPTICAL_ELEC_TRAN flag (0 = ABO possible)  */
  int32_t otr[2];   /* optical-electron orbitals (s=0,p=1,d=2,f=3)*/
  int32_t abo_ierr; /* GET_COLLISIONAL_PARAM status               */
  int32_t pad;
  double l0;        /* central wavelength [A]                     */
  double loggf, eplow, alpha, sigma;
  double sl, ll, jl, su, lu, ju;
  double elowlim, eupplim;
} orc_line;

/* One spectral region of the LINES: section (src/input_file.f90:290-366). */
#define ORC_MAXBLEND 8
typedef struct {
  int32_t nblend;                 /* number of lines in the region (>=1)   */
  int32_t line[ORC_MAXBLEND];     /* 0-based index into the line table     */
  double wdif[ORC_MAXBLEND];      /* BLENDSDIFF [mA] (0 for the main line) */
  int32_t numwave;
  int32_t pad;
  double wave_ini, dlambda;       /* [mA]                                   */
} orc_region;

/* Status codes (per column) replacing the reference STOPs. */
#define ORC_OK 0
#define ORC_CHEM_NOCONV 1
#define ORC_NAN 2

int orc_version(void);

/* Test hook: replace the abundance set (NULL restores the default). */
void orc_set_abundances(const double* abund92);

/* Partition function U_I,U_II,U_III and dlnU/dT (src/atom_database.f90:121). */
void orc_partition(int zn, double T, double out6[6]);

/* GET_RHO (src/chemical_equilibrium.f90:165-278).  nelec is in/out (the
 * warm-start chain).  out = {nhyd, pelec, dens, molecw, iterations}. */
int orc_get_rho(double T, double pg, double* nelec, double out5[5]);

/* OPAC_CONTINUUM (src/cont_opacity.f90:305-357); T is REAL*4 in the reference. */
double orc_opac_continuum(float T, double lambda0, double ne, double nh);

/* Parse lines_database.dat text (13- or 8-column rows, END terminated),
 * including the ABO interpolation of sigma/alpha.  Returns the row count or
 * a negative error. */
int orc_parse_lines(const char* text, orc_line* out, int maxn);

/* Zeeman pattern of one line (src/magsplit.f90:38-187).  Returns NTOT. */
int orc_zeeman(const orc_line* ln, double* shift, double* strength, int* type, int maxn);

/* Voigt/Faraday (src/voigt.f:17-98, REAL*8 build). */
void orc_voigt(int n, double a, const double* v, double* h, double* f);

/* SET_BOUNDARY + OLD_ANALYTICAL_SOLVER (src/rtesolver.f90:163-187,
 * :1134-1147) on given absorption matrices: eta (7, nw, nz) ETAI..RHOV in
 * cm^-1, src (nw, nz), zz (nz) km, bnd (nz) boundary flags or NULL; out
 * (4, nw) SYN1D at the top. */
void orc_rte_solve(int nz, int nw, const double* eta, const double* src, const double* zz, const int* bnd,
                   double* out);

/* HSRA continuum normalisation GAIN(4,NUMW) (src/normalization.f90:696-754). */
int orc_gain(const orc_line* lines, int nlines, const orc_region* regs, int nreg,
             float* gain /* (4,NUMW) */);

/* FORWARD1D over ncol columns (src/forward.f90:857-1029), no response
 * functions.  model is (NZ,13,ncol) REAL*4, updated in place like the
 * reference (rho, Pe, mu, tau5 and, in hydrostatic mode, Pg).  stokes is
 * (4*NUMW, ncol).  status is (ncol).  nthreads <= 0 selects all cores. */
int orc_forward(const orc_line* lines, int nlines, const orc_region* regs, int nreg,
                const float* gain, int nz, int ncol, float* model, int hydrostatic,
                double* stokes, int* status, int nthreads);

/* FORWARD1D with response functions (MRESPFUNCT): Stokes as orc_forward plus
 * the node Jacobian EQVDSYN (src/forward.f90:552-681) of every reference
 * parameter p (1 T, 2 Pg, 4 Bx, 5 By, 6 Bz, 7 v_z) with nodes[p-1] > 0 nodes
 * (nodes[p-1] == NZ gives the response function at every height).  jac is
 * (4*NUMW, NP, ncol) REAL*4 with NP = sum of nodes.  Returns NP, or -1 for an
 * unsupported parameter (3, 8) and -2 for nodes > NZ. */
int orc_forward_rf(const orc_line* lines, int nlines, const orc_region* regs, int nreg,
                   const float* gain, int nz, int ncol, float* model, int hydrostatic,
                   const int* nodes /* [8] */, double* stokes, float* jac, int* status,
                   int nthreads);

#ifdef __cplusplus
}
#endif
