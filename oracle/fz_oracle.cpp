// TEST INFRASTRUCTURE -- not part of the product.
//
// FP64 CPU restatement of the FIRTEZ-dz Stokes synthesis path.  Only tests/,
// __graft_entry__.smoke() and the cpu_baseline leg of bench.py load this
// library, and only as the checker / timed CPU baseline.
//
// Fidelity rules followed throughout:
//  * REAL*4 literals of the reference are used as their float32 images
//    (e.g. 13.595 in cont_opacity.f90:255, 0.3181818 in damping.f90:853);
//  * REAL*4 state (the atmosphere, src/atm_param.f90:14-25) is rounded to
//    float32 exactly where the reference stores it;
//  * evaluation order of the arithmetic follows the Fortran expressions;
//  * undefined values of the reference (uninitialised NELEC before the first
//    GET_RHO of a column, forward.f90:876) are defined as 0, which selects
//    the reference's own cold-start guess PG/(101 k T) (chemical_equilibrium.f90:192).
#include "fz_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../firtez-dz_b200/csrc/fz_tables.h"

namespace {

// ---------------------------------------------------------------- constants
// src/cons_param.f90:14-29
const double DPI = 3.141592653589793238462643;
const double LIGHT = 2.99792458e+10;
const double KBOL = 1.38056503e-16;
const double MELE = 9.10938215e-28;
const double QELE = 4.80320425e-10;
const double EVOLT = 1.60217656e-12;
const double MAMU = 1.66053892e-24;
const double HPLA = 6.62606957e-27;
const double GRAV = 2.7414e4;
double CSAHA1, CSAHA2, RBOHR;
double DENO_SA, DENO_SAM;   // src/atom_database.f90:107-112
double AB10[FZ_NELEM];      // 10**(ABUND-12)
double ABUND[FZ_NELEM];     // active abundance set (src/atom_database.f90:80-88)

void set_abund(const double* ab) {
  DENO_SA = 0.0;
  DENO_SAM = 0.0;
  for (int i = 0; i < FZ_NELEM; ++i) {
    ABUND[i] = ab ? ab[i] : fz_tab_abund[i];
    AB10[i] = std::pow(10.0, ABUND[i] - 12.0);
    DENO_SA = DENO_SA + AB10[i];
    DENO_SAM = DENO_SAM + MAMU * fz_tab_matom[i] * AB10[i];
  }
}

inline double sp(double x) { return (double)(float)x; }   // REAL*4 literal image

struct Init {
  Init() {
    CSAHA1 = std::pow(HPLA, 3.0) / std::pow(2.0 * DPI * MELE * KBOL, 3.0 / 2.0);
    CSAHA2 = EVOLT / KBOL;
    RBOHR = std::pow(HPLA, 2.0) / (4.0 * std::pow(DPI, 2.0) * MELE * std::pow(QELE, 2.0));
    set_abund(nullptr);
  }
} g_init;

// ------------------------------------------------- partition functions
// Table evaluator for src/atom_database.f90:121-1035 (pieces generated by
// oracle/gen_tables.py; pinned against a literal evaluation of the Fortran).
inline double horner(const double* c, int n, double x) {
  double r = c[n - 1];
  for (int i = n - 2; i >= 0; --i) r = c[i] + x * r;
  return r;
}

inline bool cond_holds(int cond, double th, double T, double u) {
  switch (cond) {
    case 0: return true;
    case 1: return T > th;
    case 2: return T < th;
    case 3: return T <= th;
    case 4: return T >= th;
    case 5: return u != th;
  }
  return false;
}

inline double vpiece(const fz_pf_vpiece& p, const double* var) {
  double h = horner(p.c, p.nc, var[p.var]);
  if (p.form == 1) return p.base + std::exp(h);
  if (p.form == 2) return std::max(p.clamp, h);
  return h;
}

void partition(int zn, double T, double U[3], double dU[3]) {
  const int e = zn - 1;
  const double var[3] = {T, 1.0e-3 * T, std::log(5040.0 / T)};
  for (int s = 0; s < 3; ++s) {
    const int nv = fz_tab_pf_nv[e][s];
    int act = -1;
    for (int i = 0; i < nv; ++i)
      if (cond_holds(fz_tab_pf_v[e][s][i].cond, fz_tab_pf_v[e][s][i].th, T, 0.0)) act = i;
    U[s] = act >= 0 ? vpiece(fz_tab_pf_v[e][s][act], var) : 0.0;
    double d = 0.0;
    const int nd = fz_tab_pf_nd[e][s];
    for (int i = 0; i < nd; ++i) {
      const fz_pf_dpiece& p = fz_tab_pf_d[e][s][i];
      const double uref = p.ref >= 0 ? vpiece(fz_tab_pf_v[e][s][p.ref], var) : U[s];
      if (!cond_holds(p.cond, p.th, T, uref)) continue;
      double h = horner(p.c, p.nc, var[p.var]) * p.mult;
      for (int k = 0; k < p.dx; ++k) h *= (-1.0 / T);
      if (p.ub) h *= (uref - p.base);
      for (int k = 0; k < p.up; ++k) h /= uref;
      d = h;
    }
    dU[s] = d;
  }
}

// ------------------------------------------------ chemical equilibrium
// SHORT_PRE_ION_CALC_TEMPRHO, src/chemical_equilibrium.f90:1601-1652
void short_pre(double T, double* a1, double* a2) {
  const double lamelec = CSAHA1 * std::pow(T, -3.0 / 2.0);
  for (int i = 0; i < FZ_NELEM; ++i) {
    double U[3], dU[3];
    partition(i + 1, T, U, dU);
    double e1 = CSAHA2 * fz_tab_xi[i] / T;
    double e2 = CSAHA2 * fz_tab_xii[i] / T;
    if (e1 > 0.0) e1 = std::min(e1, 650.0);
    if (e1 < 0.0) e1 = std::max(e1, -650.0);
    if (e2 > 0.0) e2 = std::min(e2, 650.0);
    if (e2 < 0.0) e2 = std::max(e2, -650.0);
    e1 = std::exp(e1);
    e2 = std::exp(e2);
    a1[i] = (U[0] / (2.0 * U[1])) * lamelec * e1;
    a2[i] = (U[1] / (2.0 * U[2])) * lamelec * e2;
  }
}

struct Rho {
  double nhyd, pelec, dens, molecw;
  int iters;
  int status;
};

// GET_RHO, src/chemical_equilibrium.f90:165-278
Rho get_rho(double T, double PG, double& nelec) {
  Rho r{};
  double nhyd = 0.0;
  if (nelec != nelec) nelec = 0.0;
  if (nelec < 1.0) nelec = PG / (101.0 * KBOL * T);
  double pelec = nelec * KBOL * T;
  if (pelec > PG) nelec = (PG * 0.5) / (KBOL * T);
  double a1[FZ_NELEM], a2[FZ_NELEM];
  short_pre(T, a1, a2);
  double err = 1.0;
  int iter = 1;
  double nnew = nelec, nold = nelec;
  while (err > 1.0e-4 && iter <= 100 && nhyd >= 0.0) {
    nold = nnew;
    const double nume = PG - nnew * KBOL * T;
    nhyd = nume / (DENO_SA * KBOL * T);
    // SHORT_ION_CALC_TEMPRHO, :1659-1701, with NE = nnew
    const double ne = nnew;
    double vni1 = 0, vniii1 = 0, s2 = 0.0, s3 = 0.0;
    for (int i = 0; i < FZ_NELEM; ++i) {
      const double vnt = nhyd * AB10[i];
      const double vni = vnt / (1.0 + (1.0 / (ne * a1[i])) * (1.0 + (1.0 / (ne * a2[i]))));
      const double vnii = vnt / (ne * a1[i] + 1.0 + (1.0 / (ne * a2[i])));
      const double vniii = vnt / (1.0 + ne * a2[i] * (ne * a1[i] + 1.0));
      if (i == 0) {
        vni1 = vni;
        vniii1 = vniii;
      } else {
        s2 = s2 + vnii;
        s3 = s3 + vniii;
      }
    }
    double est = vniii1 - vni1;
    est = est + s2 + s3;
    nnew = (std::max(est, 0.0) + nold) / 2.0;
    err = std::fabs((nnew - nold) / nnew);
    iter = iter + 1;
  }
  r.status = ORC_OK;
  if (iter >= 100 || nhyd < 0.0) r.status = ORC_CHEM_NOCONV;
  nelec = nnew;
  const double nume = PG - nelec * KBOL * T;
  nhyd = nume / (DENO_SA * KBOL * T);
  const double dens = nhyd * DENO_SAM + nelec * MELE;
  const double molecw = ((dens * KBOL * T) / MAMU) * std::pow(PG, -1.0);
  if (nhyd != nhyd || nnew != nnew) r.status = ORC_NAN;
  if (nelec < 0.0 || nhyd <= 0.0) r.status = ORC_CHEM_NOCONV;
  r.nhyd = nhyd;
  r.pelec = pelec;   // the reference returns the pressure of the initial guess
  r.dens = dens;
  r.molecw = molecw;
  r.iters = iter;
  return r;
}

// ION_CALC_TEMPX, src/chemical_equilibrium.f90:1511-1597 (value only)
double ion_calc_tempx(int zn, int ion, double T, double ne, double n) {
  double U[3], dU[3];
  partition(zn, T, U, dU);
  const double lamelec = CSAHA1 * std::pow(T, -3.0 / 2.0);
  double e1 = CSAHA2 * fz_tab_xi[zn - 1] / T;
  double e2 = CSAHA2 * fz_tab_xii[zn - 1] / T;
  if (e1 > 0.0) e1 = std::min(e1, 650.0);
  if (e1 < 0.0) e1 = std::max(e1, -650.0);
  if (e2 > 0.0) e2 = std::min(e2, 650.0);
  if (e2 < 0.0) e2 = std::max(e2, -650.0);
  e1 = std::exp(e1);
  e2 = std::exp(e2);
  const double al1 = (U[0] / (2.0 * U[1])) * lamelec * e1;
  const double al2 = (U[1] / (2.0 * U[2])) * lamelec * e2;
  const double deno = std::pow(ne, 2.0) * al1 * al2 + ne * al2 + 1.0;
  double nume = 1.0;
  if (ion == 1) nume = std::pow(ne, 2.0) * al1 * al2;
  if (ion == 2) nume = ne * al2;
  return n * nume / deno;
}

// ------------------------------------------------------ continuum opacity
// src/cont_opacity.f90:48-357
double hminus_ff(double T, double ne, double l0) {
  static const double A1[6] = {0, 2483.346, -3449.889, 2200.04, -696.271, 88.283};
  static const double B1[6] = {0, 285.827, -1158.382, 2427.719, -1841.4, 444.517};
  static const double C1[6] = {0, -2054.291, 8746.523, -13651.105, 8624.97, -1863.864};
  static const double D1[6] = {0, 2827.776, -11485.632, 16755.524, -10051.53, 2095.288};
  static const double E1[6] = {0, -1341.537, 5303.609, -7510.494, 4400.067, -901.788};
  static const double F1[6] = {0, 208.952, -812.939, 1132.738, -655.02, 132.985};
  static const double A2[4] = {518.1021, 473.2636, -482.2089, 115.5291};
  static const double B2[4] = {-734.8666, 1443.4137, -737.1616, 169.6374};
  static const double C2[4] = {1021.1775, -1977.3395, 1096.8827, -245.649};
  static const double D2[4] = {-479.0721, 922.3575, -521.1341, 114.243};
  static const double E2[4] = {93.1373, -178.9275, 101.7963, -21.9972};
  static const double F2[4] = {-6.4285, 12.36, -7.0571, 1.5097};
  const double lm = l0 / 1e4;
  const double th = 5040.0 / T;
  double part1;
  if (lm < 0.3645) {
    double c[4];
    for (int i = 0; i < 4; ++i)
      c[i] = A2[i] * std::pow(lm, 2.0) + B2[i] + C2[i] / lm + D2[i] / std::pow(lm, 2.0) +
             E2[i] / std::pow(lm, 3.0) + F2[i] / std::pow(lm, 4.0);
    part1 = c[0] * th + c[1] * std::pow(th, 1.5) + c[2] * std::pow(th, 2.0) + c[3] * std::pow(th, 2.5);
  } else {
    double c[6];
    for (int i = 0; i < 6; ++i)
      c[i] = A1[i] * std::pow(lm, 2.0) + B1[i] + C1[i] / lm + D1[i] / std::pow(lm, 2.0) +
             E1[i] / std::pow(lm, 3.0) + F1[i] / std::pow(lm, 4.0);
    part1 = c[0] * th + c[1] * std::pow(th, 1.5) + c[2] * std::pow(th, 2.0) + c[3] * std::pow(th, 2.5) +
            c[4] * std::pow(th, 3.0) + c[5] * std::pow(th, 3.5);
  }
  return 1e-29 * part1 * KBOL * ne * T;
}

double hminus_bf(double T, double ne, double l0) {
  const double LAMBDAP = 1.6419, CTE = 0.75e-18;
  const double ALPHA = (HPLA * LIGHT / KBOL) * 1e4;
  static const double CC[6] = {152.519, 49.534, -118.858, 92.536, -34.194, 4.982};
  const double lm = l0 / 1e4;
  if (!(lm < LAMBDAP)) return 0.0;
  const double com = 1.0 / lm - 1.0 / LAMBDAP;
  double sigma = CC[0] + CC[1] * std::pow(com, 0.5) + CC[2] * com + CC[3] * std::pow(com, 1.5) +
                 CC[4] * std::pow(com, 2.0) + CC[5] * std::pow(com, 2.5);
  sigma = CTE * sigma * std::pow(lm, 3.0) * std::pow(com, 1.5);
  const double part = std::pow(T, -2.5) * std::exp(ALPHA / (T * LAMBDAP)) * (1.0 - std::exp(-ALPHA / (T * lm)));
  return part * sigma * ne * KBOL * T;
}

double thomson(double ne, double nh) {
  const double CT = (8.0 * DPI / 3.0) * (std::pow(QELE / LIGHT, 4.0)) / std::pow(MELE, 2.0);
  return CT * (ne / nh);
}

double rayleigh_h(double l0) {
  const double c1 = 5.799e-13, c2 = 1.422e-6, c3 = 2.784;
  return (c1 + (c2 + c3 / std::pow(l0, 2.0)) / std::pow(l0, 2.0)) / std::pow(l0, 4.0);
}

double hydrogen(double T, double l0) {
  const double IOPOT = sp(13.595);
  const double C1 = sp(1e-8) * IOPOT * EVOLT / (HPLA * LIGHT);
  const double C2 = std::pow(sp(1e-8), 3.0) * 64.0 * std::pow(DPI, 4.0) * MELE * std::pow(QELE, 10.0) /
                    (3.0 * std::sqrt(3.0) * std::pow(LIGHT, 4.0) * std::pow(HPLA, 6.0));
  const double C3 = HPLA * LIGHT / (KBOL * sp(1e-8));
  const double C4 = IOPOT * EVOLT / KBOL;
  const int n0 = 1 + (int)std::floor(std::sqrt(C1 * l0));
  double sum;
  if (n0 <= 8) {
    sum = std::exp(C4 / (T * std::pow((double)n0, 2.0))) * std::pow((double)n0, -3.0);
    for (int i = n0 + 1; i <= 8; ++i)
      sum = sum + std::exp(C4 / (T * std::pow((double)i, 2.0))) * std::pow((double)i, -3.0);
    sum = sum + (0.117 + std::exp(C4 / (T * std::pow(9.0, 2.0)))) * (T / (2.0 * C4));
  } else {
    sum = (0.117 + std::exp(C4 / (T * std::pow((double)n0, 2.0)))) * (T / (2.0 * C4));
  }
  return C2 * sum * (1.0 - std::exp(-C3 / (T * l0))) * std::exp(-C4 / T) * std::pow(l0, 3.0);
}

double opac_continuum(float Tsp, double l0, double ne, double nh) {
  const double T = (double)Tsp;
  if (l0 < 1800.0) return NAN;   // HMINUS_FF STOPs below 1800 A
  const double factor = hminus_ff(T, ne, l0) + hminus_bf(T, ne, l0) + thomson(ne, nh) + rayleigh_h(l0) +
                        hydrogen(T, l0);
  return nh * factor;
}

// ------------------------------------------------------------ line opacity
// OPAC_LINE, src/line_opacity.f90:34-108 (LTE departure coefficients = 1)
double opac_line(const orc_line& ln, float Tsp, double ne, double nh) {
  const double bl = 1.0, bu = 1.0;
  const double T = (double)Tsp;
  const double n = nh * std::pow(10.0, ABUND[ln.zn - 1] - 12.0);
  const double npi = ion_calc_tempx(ln.zn, ln.ion, T, ne, n);
  double U[3], dU[3];
  partition(ln.zn, T, U, dU);
  const double upi = U[ln.ion - 1];
  const double t1 = std::sqrt(DPI) * std::pow(QELE, 2.0) / (MELE * LIGHT) * std::pow(10.0, ln.loggf) * ln.l0 * 1e-8;
  const double t2 = std::sqrt(fz_tab_matom[ln.zn - 1] * MAMU / (2.0 * KBOL * T));
  const double t3 = bl * npi / upi;
  const double t4 = std::exp(-ln.eplow * EVOLT / (KBOL * T));
  const double t5 = 1.0 - (bu / bl) * std::exp(-HPLA * LIGHT / (1.0e-8 * ln.l0 * KBOL * T));
  return t1 * t2 * t3 * t4 * t5;
}

// ------------------------------------------------------------------ damping
// REFRAX, src/atom_database.f90:1039-1074
double refrax(double w) {
  const double T = 15.0, P = 760.0, H = 0.0;
  const double s = 1.0 / std::pow(w, 2.0);
  const double r = 6.4328e-5 + 2.94981e-2 / (146.0 - s) + 2.554e-4 / (41.0 - s);
  const double y = 1.0 / (273.15 + T);
  const double alpha = 3.67e-3 + 3.3e-4 * std::exp((0.19 - w) / 0.12);
  const double wvsp = std::pow(10.0, -55.1132754 + y * (1.19551822e5 + y * (-9.70108858e7 + y * (4.12856913e10 +
                                       y * (-9.87931835e12 + y * (1.25868645e15 - 6.66885272e16 * y))))));
  const double wvp = 1.0e-2 * H * wvsp;
  return 1.0 + 1.31579e-3 * r * P / (1.0 + alpha * (T - 1.0) / (1.0 + 15.0 * alpha)) - 5.49e-8 * wvp / (1.0 + alpha * T);
}

// GET_DAMPING, src/damping.f90:842-1012 (value only)
double get_damping(const orc_line& ln, double nhyd, float Tsp) {
  const int I = ln.zn;
  const double lambda = ln.l0 * 1e-8;
  const double T8 = (double)Tsp;
  const double RAT = sp(0.3181818);
  const double V0 = 1e6;
  const double m = fz_tab_matom[I - 1], m1 = fz_tab_matom[0], m2 = fz_tab_matom[1];
  const double vdop = std::sqrt(2.0 * KBOL * T8 / (MAMU * m));
  const double grad = 0.2223 / std::pow(lambda, 2.0);           // RADIATIVE_DAMPING :1309-1319
  const double mu_h = MAMU * (m * m1) / (m + m1);
  const double mu_he = MAMU * (m * m2) / (m + m2);
  const double nhe = nhyd * std::pow(10.0, ABUND[1] - 12.0);
  double gcol;
  if (ln.sigma > 0 && ln.alpha > 0) {
    const double e1 = 2.0 - ln.alpha / 2.0;
    const double e2 = (1.0 - ln.alpha) / 2.0;
    const double gammaf =
        1.0 + (-0.5748646 + (0.9512363 + (-0.6998588 + (0.4245549 - 0.1010678 * e1) * e1) * e1) * e1) * e1;
    double beta = std::pow(4.0 / DPI, ln.alpha / 2.0) * gammaf * std::pow(V0, ln.alpha) *
                  (ln.sigma * std::pow(RBOHR, 2.0)) * std::pow(8.0 * KBOL / DPI, e2);
    beta = 2.0 * beta;
    gcol = beta * std::pow(T8, e2) * (nhyd * std::pow(mu_h, -e2) + RAT * nhe * std::pow(mu_he, -e2));
  } else {
    double rindex = sp(1.0004);
    if (lambda * 1e8 >= 1800.0) rindex = refrax(lambda * 1e4);
    const double lvac = rindex * lambda;
    const double epupp = ln.eplow + (HPLA * LIGHT / lvac) / EVOLT;
    double ed1, ed2, chyd;
    if (ln.ion == 1) {
      ed1 = std::max(fz_tab_xi[I - 1] - epupp - fz_tab_xi[I - 1] * (double)(float)(ln.ion - 1), 1.0);
      ed2 = std::max(fz_tab_xi[I - 1] - ln.eplow - fz_tab_xi[I - 1] * (double)(float)(ln.ion - 1), 3.0);
      chyd = 1.0;
    } else {
      ed1 = std::max(fz_tab_xii[I - 1] - epupp - fz_tab_xi[I - 1] * (double)(float)(ln.ion - 1), 1.0);
      ed2 = std::max(fz_tab_xii[I - 1] - ln.eplow - fz_tab_xi[I - 1] * (double)(float)(ln.ion - 1), 3.0);
      chyd = sp(1.741);
    }
    chyd = chyd * 17.0 * std::pow(8.0 * KBOL / DPI, 0.3);
    chyd = chyd * std::pow(std::pow(10.0, -30.5325) * (1.0 / std::pow(ed1, 2.0) - 1.0 / std::pow(ed2, 2.0)), 0.4);
    const double chydp = chyd * (nhyd * std::pow(mu_h, -0.3) + nhe * std::pow(mu_he, -0.3));
    gcol = chydp * std::pow((double)Tsp, 0.3);
  }
  return (grad + gcol) * lambda / (4.0 * DPI * vdop);
}

// ------------------------------------------------------------------- Voigt
// src/voigt.f:17-98 compiled with -fdefault-real-8: complex(8) arithmetic,
// gfortran complex division with range reduction (Smith).
inline std::complex<double> cdiv(std::complex<double> a, std::complex<double> b) {
  const double ar = a.real(), ai = a.imag(), br = b.real(), bi = b.imag();
  if (std::fabs(br) >= std::fabs(bi)) {
    const double r = bi / br, den = br + bi * r;
    return {(ar + ai * r) / den, (ai - ar * r) / den};
  }
  const double r = br / bi, den = br * r + bi;
  return {(ar * r + ai) / den, (ai * r - ar) / den};
}
inline std::complex<double> cmul(std::complex<double> a, std::complex<double> b) {
  return {a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real()};
}

void voigt1(double a, double g, double& H, double& Fo) {
  static const double A0 = 122.607931777104326, A1 = 214.382388694706425, A2 = 181.928533092181549,
                      A3 = 93.155580458138441, A4 = 30.180142196210589, A5 = 5.912626209773153,
                      A6 = .564189583562615, B0 = 122.60793177387535, B1 = 352.730625110963558,
                      B2 = 457.334478783897737, B3 = 348.703917719495792, B4 = 170.354001821091472,
                      B5 = 53.992906912940207, B6 = 10.479857114260399;
  static const double XD[28] = {.1, .2, .3, .4, .5, .6, .7, .8, .9, 1., 1.2, 1.4, 1.6, 1.8,
                                 2., 3., 4., 5., 6., 7., 8., 9., 10., 12., 14., 16., 18., 20.};
  static const double YD[28] = {9.9335991E-02, 1.9475104E-01, 2.8263167E-01, 3.5994348E-01, 4.2443639E-01,
                                4.7476321E-01, 5.1050407E-01, 5.3210169E-01, 5.4072434E-01, 5.3807950E-01,
                                5.0727350E-01, 4.5650724E-01, 3.9993989E-01, 3.4677279E-01, 3.0134040E-01,
                                1.7827103E-01, 1.2934799E-01, 1.0213407E-01, 8.4542692E-02, 7.2180972E-02,
                                6.3000202E-02, 5.5905048E-02, 5.0253846E-02, 4.1812878E-02, 3.5806101E-02,
                                3.1311397E-02, 2.7820844E-02, 2.5031367E-02};
  const int sg = g < 0 ? -1 : 1;
  const double v = sg * g;
  double F;
  if (a == 0.0) {
    const double v2 = v * v;
    H = std::exp(-v2);
    double D;
    if (!(v > XD[0])) {
      D = v * (1. - .66666667 * v2);
    } else if (!(v > XD[27])) {
      int k = 27;
      for (int i = 2; i <= 27; ++i) {
        if (XD[i - 1] < v) continue;
        k = i;
        break;
      }
      const int kk = k - 1, kkk = k + 1;
      const double d1 = v - XD[kk - 1], d2 = v - XD[k - 1], d3 = v - XD[kkk - 1];
      const double d12 = XD[kk - 1] - XD[k - 1], d13 = XD[kk - 1] - XD[kkk - 1], d23 = XD[k - 1] - XD[kkk - 1];
      D = YD[kk - 1] * d2 * d3 / (d12 * d13) - YD[k - 1] * d1 * d3 / (d12 * d23) + YD[kkk - 1] * d1 * d2 / (d13 * d23);
    } else {
      const double y = .5 / v;
      D = y * (1. + y / v);
    }
    F = sg * 5.641895836E-1 * D;
  } else {
    const std::complex<double> z(a, -v);
    std::complex<double> num(A6 * z.real(), A6 * z.imag());
    num += A5; num = cmul(num, z);
    num += A4; num = cmul(num, z);
    num += A3; num = cmul(num, z);
    num += A2; num = cmul(num, z);
    num += A1; num = cmul(num, z);
    num += A0;
    std::complex<double> den = z + B6;
    den = cmul(den, z); den += B5;
    den = cmul(den, z); den += B4;
    den = cmul(den, z); den += B3;
    den = cmul(den, z); den += B2;
    den = cmul(den, z); den += B1;
    den = cmul(den, z); den += B0;
    const std::complex<double> w = cdiv(num, den);
    H = w.real();
    F = .5 * sg * w.imag();
  }
  Fo = F * 2.0;
}

// ------------------------------------------------------------------ Zeeman
// ZEEMAN_COMP, src/magsplit.f90:38-187
struct Zeeman {
  int n;
  double shift[64], strength[64];
  int type[64];
};

Zeeman zeeman(const orc_line& ln) {
  Zeeman z{};
  const double jl = ln.jl, ju = ln.ju;
  const int ntot = (int)(2 * std::min(jl, ju) + 1) + 2 * (int)(jl + ju);
  const int dj = (int)(ju - jl);
  const double glow = jl != 0 ? 1.5 + (ln.sl * (ln.sl + 1.0) - ln.ll * (ln.ll + 1.0)) / (2.0 * jl * (jl + 1.0)) : 0.0;
  const double gupp = ju != 0 ? 1.5 + (ln.su * (ln.su + 1.0) - ln.lu * (ln.lu + 1.0)) / (2.0 * ju * (ju + 1.0)) : 0.0;
  const int nmjl = (int)(2 * jl + 1), nmju = (int)(2 * ju + 1);
  int count = 0;
  for (int j = 1; j <= nmjl; ++j) {
    const double ml = (double)(j - 1.0 - jl);
    for (int k = 1; k <= nmju; ++k) {
      const double mu = (double)(k - 1.0 - ju);
      const int dm = (int)(mu - ml);
      if (std::abs(dm) > 1) continue;
      const double dl = (double)(float)(4.66685e-10 * (ml * glow - mu * gupp) * std::pow(ln.l0, 2));
      double s = 0.0;
      if (dj == -1) {
        if (dm == -1) s = (jl + mu) * (ju + mu + 2.0);
        if (dm == 0) s = 2.0 * (std::pow(jl, 2.0) - std::pow(mu, 2.0));
        if (dm == 1) s = (jl - mu) * (ju - mu + 2.0);
      } else if (dj == 0) {
        if (dm == -1) s = (ju - mu) * (ju + mu + 1.0);
        if (dm == 0) s = 2.0 * std::pow(mu, 2.0);
        if (dm == 1) s = (ju + mu) * (ju - mu + 1.0);
      } else if (dj == 1) {
        if (dm == -1) s = (ju - mu) * (jl - mu);
        if (dm == 0) s = 2.0 * (std::pow(ju, 2.0) - std::pow(mu, 2.0));
        if (dm == 1) s = (ju + mu) * (jl + mu);
      }
      z.type[count] = dm;
      z.shift[count] = dl;
      z.strength[count] = s;
      ++count;
    }
  }
  (void)ntot;
  z.n = count;
  double spi = 0, ssr = 0, ssb = 0;
  for (int j = 0; j < count; ++j) {
    if (z.type[j] == -1) ssr = ssr + z.strength[j];
    if (z.type[j] == 0) spi = spi + z.strength[j];
    if (z.type[j] == 1) ssb = ssb + z.strength[j];
  }
  for (int j = 0; j < count; ++j) {
    if (z.type[j] == -1) z.strength[j] = z.strength[j] / ssr;
    if (z.type[j] == 0) z.strength[j] = z.strength[j] / spi;
    if (z.type[j] == 1) z.strength[j] = z.strength[j] / ssb;
  }
  return z;
}

// ----------------------------------------------------- synthesis set-up
struct Setup {
  std::vector<orc_line> lines;
  std::vector<orc_region> regs;
  std::vector<Zeeman> zee;     // per line
  int numw = 0;
  std::vector<int> pini;       // PIXEL_INI (0-based)
  std::vector<double> wave;    // WAVE [mA] (src/pre_post_duties.f90:592-621)
  std::vector<int> regof;      // region of each wavelength
};

Setup make_setup(const orc_line* lines, int nlines, const orc_region* regs, int nreg) {
  Setup s;
  s.lines.assign(lines, lines + nlines);
  s.regs.assign(regs, regs + nreg);
  for (int i = 0; i < nlines; ++i) s.zee.push_back(zeeman(lines[i]));
  int p = 0;
  for (int r = 0; r < nreg; ++r) {
    s.pini.push_back(p);
    for (int j = 0; j < regs[r].numwave; ++j) {
      s.wave.push_back(regs[r].wave_ini + regs[r].dlambda * (double)j);
      s.regof.push_back(r);
    }
    p += regs[r].numwave;
  }
  s.numw = p;
  return s;
}

// SOURCE_FUNCTION, src/rtesolver.f90:1008-1035 (LTE)
inline double source_function(const Setup& s, int l, double T) {
  const int m = s.regof[l];
  double w = s.lines[s.regs[m].line[0]].l0 + s.wave[l] / 1.0e3;
  w = w * 1e-8;
  return 2.0 * HPLA * std::pow(LIGHT, 2.0) / std::pow(w, 5.0) *
         (1.0 / ((1.0 / 1.0) * std::exp(HPLA * LIGHT / (w * KBOL * T)) - 1.0));
}

struct AbsMat {
  std::vector<double> ei, eq, eu, ev, rq, ru, rv;
  void resize(int n) {
    ei.assign(n, 0); eq.assign(n, 0); eu.assign(n, 0); ev.assign(n, 0);
    rq.assign(n, 0); ru.assign(n, 0); rv.assign(n, 0);
  }
};

// GET_ABS_MAT_WODEV + ABS_MAT_FIRST_STEP/END_STEP,
// src/absorption_matrix.f90:293-845 and :849-1715
void abs_mat(const Setup& s, AbsMat& A, int L, int B, double kc, double klin, double damp, float Tk,
             float bx, float by, float bz, float vz) {
  const orc_region& rg = s.regs[L];
  const int idl = rg.line[B];
  const orc_line& ln = s.lines[idl];
  const int p0 = s.pini[L], nw = rg.numwave;
  // FIRST_STEP: keep the previous content (blends), zero the region
  std::vector<double> iei(A.ei.begin() + p0, A.ei.begin() + p0 + nw), ieq(A.eq.begin() + p0, A.eq.begin() + p0 + nw),
      ieu(A.eu.begin() + p0, A.eu.begin() + p0 + nw), iev(A.ev.begin() + p0, A.ev.begin() + p0 + nw),
      irq(A.rq.begin() + p0, A.rq.begin() + p0 + nw), iru(A.ru.begin() + p0, A.ru.begin() + p0 + nw),
      irv(A.rv.begin() + p0, A.rv.begin() + p0 + nw);
  if (B == 0) {
    std::fill(iei.begin(), iei.end(), 0.0); std::fill(ieq.begin(), ieq.end(), 0.0);
    std::fill(ieu.begin(), ieu.end(), 0.0); std::fill(iev.begin(), iev.end(), 0.0);
    std::fill(irq.begin(), irq.end(), 0.0); std::fill(iru.begin(), iru.end(), 0.0);
    std::fill(irv.begin(), irv.end(), 0.0);
  }
  for (int j = 0; j < nw; ++j) {
    A.ei[p0 + j] = 0; A.eq[p0 + j] = 0; A.eu[p0 + j] = 0; A.ev[p0 + j] = 0;
    A.rq[p0 + j] = 0; A.ru[p0 + j] = 0; A.rv[p0 + j] = 0;
  }
  const double T = (double)Tk;
  const double vdop = std::sqrt(2.0 * KBOL * T / (fz_tab_matom[ln.zn - 1] * MAMU));
  const double dldop = 1e3 * (vdop * ln.l0 / LIGHT);
  const double bbx = bx, bby = by, bbz = bz;
  const double bbx2 = std::pow(bbx, 2.0), bby2 = std::pow(bby, 2.0), bbz2 = std::pow(bbz, 2.0);
  const double bx2mby2 = bbx2 - bby2, bx2pby2 = bbx2 + bby2;
  const double bf2 = std::pow(bbx, 2.0) + std::pow(bby, 2.0) + std::pow(bbz, 2.0);
  const double bf = std::sqrt(bf2);
  double cosg = 0, cgf = 1, sgf = 1, c2p = 0, s2p = 0;
  if (bf > 0) {
    cosg = bbz / bf;
    cgf = 1 + bbz2 / bf2;
    sgf = 1 - bbz2 / bf2;
  }
  if (bbx != 0 || bby != 0) {
    c2p = bx2mby2 / bx2pby2;
    s2p = 2. * bbx * bby / bx2pby2;
  }
  const Zeeman& zc = s.zee[idl];
  const double dlv = -1e3 * ln.l0 * (double)vz / LIGHT;
  const double wdif = rg.wdif[B];
  std::vector<double> uu(nw), hh(nw), ff(nw);
  for (int m = 0; m < zc.n; ++m) {
    const double dlb = zc.shift[m] * bf;
    for (int j = 0; j < nw; ++j) uu[j] = (s.wave[p0 + j] - wdif + dlb + dlv) / dldop;
    for (int j = 0; j < nw; ++j) voigt1(damp, uu[j], hh[j], ff[j]);
    const double st = zc.strength[m];
    for (int j = 0; j < nw; ++j) {
      const double shh = st * hh[j], sff = st * ff[j];
      const int q = p0 + j;
      if (zc.type[m] == -1) {
        A.ei[q] = A.ei[q] + 0.25 * shh * cgf;
        A.eq[q] = A.eq[q] - 0.25 * shh * sgf * c2p;
        A.eu[q] = A.eu[q] - 0.25 * shh * sgf * s2p;
        A.ev[q] = A.ev[q] + 0.5 * shh * cosg;
        A.rq[q] = A.rq[q] - 0.25 * sff * sgf * c2p;
        A.ru[q] = A.ru[q] - 0.25 * sff * sgf * s2p;
        A.rv[q] = A.rv[q] + 0.5 * sff * cosg;
      } else if (zc.type[m] == 0) {
        A.ei[q] = A.ei[q] + 0.5 * shh * sgf;
        A.eq[q] = A.eq[q] + 0.5 * shh * sgf * c2p;
        A.eu[q] = A.eu[q] + 0.5 * shh * sgf * s2p;
        A.rq[q] = A.rq[q] + 0.5 * sff * sgf * c2p;
        A.ru[q] = A.ru[q] + 0.5 * sff * sgf * s2p;
      } else {
        A.ei[q] = A.ei[q] + 0.25 * shh * cgf;
        A.eq[q] = A.eq[q] - 0.25 * shh * sgf * c2p;
        A.eu[q] = A.eu[q] - 0.25 * shh * sgf * s2p;
        A.ev[q] = A.ev[q] - 0.5 * shh * cosg;
        A.rq[q] = A.rq[q] - 0.25 * sff * sgf * c2p;
        A.ru[q] = A.ru[q] - 0.25 * sff * sgf * s2p;
        A.rv[q] = A.rv[q] - 0.5 * sff * cosg;
      }
    }
  }
  for (int j = 0; j < nw; ++j) {
    const int q = p0 + j;
    A.ei[q] = kc + klin * A.ei[q];
    A.ev[q] = klin * A.ev[q];
    A.eq[q] = klin * A.eq[q];
    A.eu[q] = klin * A.eu[q];
    A.rv[q] = klin * A.rv[q];
    A.rq[q] = klin * A.rq[q];
    A.ru[q] = klin * A.ru[q];
    // END_STEP
    if (B == 0) A.ei[q] = A.ei[q] + iei[j];
    else A.ei[q] = (A.ei[q] - kc) + iei[j];
    A.eq[q] = A.eq[q] + ieq[j];
    A.eu[q] = A.eu[q] + ieu[j];
    A.ev[q] = A.ev[q] + iev[j];
    A.rq[q] = A.rq[q] + irq[j];
    A.ru[q] = A.ru[q] + iru[j];
    A.rv[q] = A.rv[q] + irv[j];
  }
}

// EVOL_OPERATOR (value part), src/rtesolver.f90:269-473
bool big(double x) { return x == x + 1.0; }

void evol_operator(const AbsMat& A, int l, double dz, double O[4][4]) {
  double ei = A.ei[l], eq = A.eq[l], eu = A.eu[l], ev = A.ev[l], rq = A.rq[l], ru = A.ru[l], rv = A.rv[l];
  bool imat = big(ei) || big(eq) || big(eu) || big(ev) || big(rq) || big(ru) || big(rv);
  if (imat) ei = eq = eu = ev = rq = ru = rv = 1e15;
  double M2[4][4] = {}, M3[4][4] = {}, M4[4][4] = {};
  double sigma = 0.;
  const double eta2 = std::pow(eq, 2.) + std::pow(eu, 2.) + std::pow(ev, 2.);
  const double rho2 = std::pow(rq, 2.) + std::pow(ru, 2.) + std::pow(rv, 2.);
  const double er = eq * rq + eu * ru + ev * rv;
  double rpart = std::sqrt((std::pow(eta2 - rho2, 2.)) / 4. + std::pow(er, 2.)) + (eta2 - rho2) / 2.;
  const double l1 = std::sqrt(rpart);
  rpart = std::sqrt((std::pow(eta2 - rho2, 2.)) / 4. + std::pow(er, 2.)) - (eta2 - rho2) / 2.;
  const double l2 = std::sqrt(rpart);
  if (er > 0) sigma = 1.;
  if (er < 0) sigma = -1.;
  const double theta = 2. * std::sqrt((std::pow(eta2 - rho2, 2.)) / 4. + std::pow(er, 2.));
  // Fortran (row,col) 1-based -> [row-1][col-1]
  M2[1][0] = l2 * eq - sigma * l1 * rq;
  M2[2][0] = l2 * eu - sigma * l1 * ru;
  M2[3][0] = l2 * ev - sigma * l1 * rv;
  M2[0][1] = M2[1][0];
  M2[2][1] = sigma * l1 * ev + l2 * rv;
  M2[3][1] = -sigma * l1 * eu - l2 * ru;
  M2[0][2] = M2[2][0];
  M2[1][2] = -M2[2][1];
  M2[3][2] = sigma * l1 * eq + l2 * rq;
  M2[0][3] = M2[3][0];
  M2[1][3] = -M2[3][1];
  M2[2][3] = -M2[3][2];
  M3[1][0] = l1 * eq + sigma * l2 * rq;
  M3[2][0] = l1 * eu + sigma * l2 * ru;
  M3[3][0] = l1 * ev + sigma * l2 * rv;
  M3[0][1] = M3[1][0];
  M3[2][1] = -sigma * l2 * ev + l1 * rv;
  M3[3][1] = sigma * l2 * eu - l1 * ru;
  M3[0][2] = M3[2][0];
  M3[1][2] = -M3[2][1];
  M3[3][2] = -sigma * l2 * eq + l1 * rq;
  M3[0][3] = M3[3][0];
  M3[1][3] = -M3[3][1];
  M3[2][3] = -M3[3][2];
  M4[0][0] = (eta2 + rho2) / 2.;
  M4[1][0] = ev * ru - eu * rv;
  M4[2][0] = eq * rv - ev * rq;
  M4[3][0] = eu * rq - eq * ru;
  M4[0][1] = -M4[1][0];
  M4[1][1] = std::pow(eq, 2.) + std::pow(rq, 2.) - M4[0][0];
  M4[2][1] = eq * eu + rq * ru;
  M4[3][1] = ev * eq + rv * rq;
  M4[0][2] = -M4[2][0];
  M4[1][2] = M4[2][1];
  M4[2][2] = std::pow(eu, 2.) + std::pow(ru, 2.) - M4[0][0];
  M4[3][2] = eu * ev + ru * rv;
  M4[0][3] = -M4[3][0];
  M4[1][3] = M4[3][1];
  M4[2][3] = M4[3][2];
  M4[3][3] = std::pow(ev, 2.) + std::pow(rv, 2.) - M4[0][0];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      M2[i][j] = M2[i][j] / theta;
      M3[i][j] = M3[i][j] / theta;
      M4[i][j] = 2. * M4[i][j] / theta;
    }
  if (theta == 0) {
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) M2[i][j] = M3[i][j] = M4[i][j] = 0.0;
  }
  double ch = std::cosh(l1 * dz), sh = std::sinh(l1 * dz);
  if (big(ch)) ch = 1e15;
  if (big(sh)) sh = 1e15;
  const double c2 = std::cos(l2 * dz), s2 = std::sin(l2 * dz);
  const double ex = std::exp(-ei * dz);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      const double m1 = (i == j) ? 1.0 : 0.0;
      O[i][j] = ex * (0.5 * (ch + c2) * m1 - s2 * M2[i][j] - sh * M3[i][j] + 0.5 * (ch - c2) * M4[i][j]);
    }
  if (imat)
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) O[i][j] = (i == j) ? 1.0 : 0.0;
}

struct Col {
  float* m;   // MODEL(NZ,13)
  int nz;
  float& T(int k) { return m[0 * nz + k]; }
  float& PG(int k) { return m[1 * nz + k]; }
  float& RHO(int k) { return m[2 * nz + k]; }
  float& PEL(int k) { return m[3 * nz + k]; }
  float& MW(int k) { return m[4 * nz + k]; }
  float& BX(int k) { return m[5 * nz + k]; }
  float& BY(int k) { return m[6 * nz + k]; }
  float& BZ(int k) { return m[7 * nz + k]; }
  float& VZ(int k) { return m[10 * nz + k]; }
  float& TAU(int k) { return m[11 * nz + k]; }
  double Z(int k) { return (double)m[12 * nz + k]; }
};

// RK4_INTEGRATION_LOG (from the top), src/hydrostatic_tools.f90:150-222 with
// RK4_LOG :350-396 and RK4_SOLVE_LOG :53-71
int rk4_integration_log(Col& c, std::vector<double>& vnhyd) {
  const int nz = c.nz;
  int st = ORC_OK;
  std::vector<double> pg8(nz, 0), rho8(nz, 0), pel8(nz, 0), mw8(nz, 0), t8(nz);
  for (int k = 0; k < nz; ++k) t8[k] = (double)c.T(k);
  pg8[nz - 1] = std::log((double)c.PG(nz - 1));
  rho8[nz - 1] = c.RHO(nz - 1);
  pel8[nz - 1] = c.PEL(nz - 1);
  double nelec = pel8[nz - 1] / KBOL / t8[nz - 1];
  mw8[nz - 1] = c.MW(nz - 1);
  double t0 = c.Z(nz - 1) * 1000.0 * 100.0;
  double u0 = pg8[nz - 1];
  Rho r = get_rho(t8[nz - 1], std::exp(u0), nelec);
  if (r.status) st = r.status;
  rho8[nz - 1] = r.dens;
  pel8[nz - 1] = r.pelec;
  mw8[nz - 1] = r.molecw;
  vnhyd[nz - 1] = r.nhyd;
  auto dpdz = [&](double y, double tem) {
    Rho q = get_rho(tem, std::exp(y), nelec);
    if (q.status) st = q.status;
    return -q.molecw * MAMU * GRAV / (KBOL * tem);
  };
  for (int k = nz - 2; k >= 0; --k) {
    const double dz = (c.Z(k) - c.Z(k + 1)) * 1000.0 * 100.0;
    const double t1 = t0 + dz;
    const double tm0 = t8[k + 1], tm1 = t8[k];
    double tem = tm0;
    const double k1 = dpdz(u0, tem) * dz;
    const double it1 = t0 + dz / 2.0;
    const double iy1 = u0 + k1 / 2.0;
    tem = tm0 / dz * (t0 + dz - it1) + tm1 / dz * (it1 - t0);
    const double k2 = dpdz(iy1, tem) * dz;
    const double iy2 = u0 + k2 / 2.0;
    const double k3 = dpdz(iy2, tem) * dz;
    const double iy3 = u0 + k3;
    tem = tm1;
    const double k4 = dpdz(iy3, tem) * dz;
    const double u1 = u0 + 1.0 / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4);
    Rho q = get_rho(t8[k], std::exp(u1), nelec);
    if (q.status) st = q.status;
    rho8[k] = q.dens;
    pel8[k] = q.pelec;
    mw8[k] = q.molecw;
    pg8[k] = u1;
    vnhyd[k] = q.nhyd;
    u0 = u1;
    t0 = t1;
  }
  for (int k = 0; k < nz; ++k) {
    c.PG(k) = (float)std::exp(pg8[k]);
    c.RHO(k) = (float)rho8[k];
    c.PEL(k) = (float)pel8[k];
    c.MW(k) = (float)mw8[k];
  }
  return st;
}

// RK4_INTEGRATION_LOG_LTAUM05 -> RK4_INTEGRATION_LOG_MED
// (src/hydrostatic_tools.f90:226-346): HE anchored at IZ = MINLOC(ABS(TAU5))
// (the first least |log tau5|, from the input model), Pg(IZ) kept, RK4 up
// to the top, then from IZ down to the bottom with NELEC restarted from the
// anchor's Pe.
int rk4_integration_log_med(Col& c, std::vector<double>& vnhyd) {
  const int nz = c.nz;
  int iz = 0;
  for (int k = 1; k < nz; ++k)
    if (std::fabs(c.TAU(k)) < std::fabs(c.TAU(iz))) iz = k;
  int st = ORC_OK;
  std::vector<double> pg8(nz, 0), rho8(nz, 0), pel8(nz, 0), mw8(nz, 0), t8(nz);
  for (int k = 0; k < nz; ++k) t8[k] = (double)c.T(k);
  pg8[iz] = std::log((double)c.PG(iz));
  pel8[iz] = c.PEL(iz);
  double nelec = pel8[iz] / KBOL / t8[iz];
  Rho r = get_rho(t8[iz], std::exp(pg8[iz]), nelec);
  if (r.status) st = r.status;
  rho8[iz] = r.dens;
  pel8[iz] = r.pelec;
  mw8[iz] = r.molecw;
  vnhyd[iz] = r.nhyd;
  auto dpdz = [&](double y, double tem) {
    Rho q = get_rho(tem, std::exp(y), nelec);
    if (q.status) st = q.status;
    return -q.molecw * MAMU * GRAV / (KBOL * tem);
  };
  // one RK4_LOG step from height kf to the adjacent kt, then GET_RHO at kt
  auto step = [&](int kf, int kt, double& t0, double& u0) {
    const double dz = (c.Z(kt) - c.Z(kf)) * 1000.0 * 100.0;
    const double t1 = t0 + dz;
    const double tm0 = t8[kf], tm1 = t8[kt];
    const double k1 = dpdz(u0, tm0) * dz;
    const double it1 = t0 + dz / 2.0;
    const double tmid = tm0 / dz * (t0 + dz - it1) + tm1 / dz * (it1 - t0);
    const double k2 = dpdz(u0 + k1 / 2.0, tmid) * dz;
    const double k3 = dpdz(u0 + k2 / 2.0, tmid) * dz;
    const double k4 = dpdz(u0 + k3, tm1) * dz;
    const double u1 = u0 + 1.0 / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4);
    Rho q = get_rho(t8[kt], std::exp(u1), nelec);
    if (q.status) st = q.status;
    rho8[kt] = q.dens;
    pel8[kt] = q.pelec;
    mw8[kt] = q.molecw;
    pg8[kt] = u1;
    vnhyd[kt] = q.nhyd;
    u0 = u1;
    t0 = t1;
  };
  double t0 = c.Z(iz) * 1000.0 * 100.0, u0 = pg8[iz];
  for (int k = iz + 1; k < nz; ++k) step(k - 1, k, t0, u0);
  t0 = c.Z(iz) * 1000.0 * 100.0;
  u0 = pg8[iz];
  nelec = pel8[iz] / KBOL / t8[iz];
  for (int k = iz - 1; k >= 0; --k) step(k + 1, k, t0, u0);
  for (int k = 0; k < nz; ++k) {
    c.PG(k) = (float)std::exp(pg8[k]);
    c.RHO(k) = (float)rho8[k];
    c.PEL(k) = (float)pel8[k];
    c.MW(k) = (float)mw8[k];
  }
  return st;
}

// FORWARD1D without response functions, src/forward.f90:857-1029
int forward1d(const Setup& s, const float* gain, Col& c, int hydrostatic, double* stokes) {
  const int nz = c.nz, numw = s.numw;
  const double KC5THRESHOLD = 2.0e10;
  int st = ORC_OK;
  std::vector<double> vnhyd(nz, 0.0), vnelec(nz, 0.0), kc5(nz, 0.0);
  if (hydrostatic) {
    // 1: HYDRO_TOP (from the top); 2: anchored at log tau5 ~ 0 (HYDRO_TOP off)
    st = hydrostatic == 2 ? rk4_integration_log_med(c, vnhyd) : rk4_integration_log(c, vnhyd);
    for (int k = 0; k < nz; ++k) vnelec[k] = (double)c.PEL(k) / KBOL / (double)c.T(k);
  }
  std::vector<double> syn(4 * numw, 0.0);
  AbsMat A;
  A.resize(numw);
  const int nreg = (int)s.regs.size();
  std::vector<double> kc(nreg, 0.0);
  std::vector<double> klin(nreg * ORC_MAXBLEND, 0.0);
  double nhyd = 0.0, nelec = 0.0;
  for (int k = 0; k < nz; ++k) {
    if (!hydrostatic) {
      // GET_NHNEMU_G, src/chemical_equilibrium.f90:2391-2441
      Rho r = get_rho((double)c.T(k), (double)c.PG(k), nelec);
      if (r.status) st = r.status;
      nhyd = r.nhyd;
      c.RHO(k) = (float)r.dens;
      c.MW(k) = (float)r.molecw;
      c.PEL(k) = (float)r.pelec;
    } else {
      nhyd = vnhyd[k];
      nelec = vnelec[k];
    }
    kc5[k] = opac_continuum(c.T(k), 5000.0, nelec, nhyd);
    kc5[k] = kc5[k] / nhyd * (1.0 / MAMU);
    if (kc5[k] < KC5THRESHOLD) {
      for (int L = 0; L < nreg; ++L) {
        kc[L] = opac_continuum(c.T(k), s.lines[s.regs[L].line[0]].l0, nelec, nhyd);
        for (int B = 0; B < s.regs[L].nblend; ++B) {
          const orc_line& ln = s.lines[s.regs[L].line[B]];
          const double kl = opac_line(ln, c.T(k), nelec, nhyd);
          const double damp = get_damping(ln, nhyd, c.T(k));
          abs_mat(s, A, L, B, kc[L], kl, damp, c.T(k), c.BX(k), c.BY(k), c.BZ(k), c.VZ(k));
        }
      }
    }
    for (int l = 0; l < numw; ++l) {
      const double S = source_function(s, l, (double)c.T(k));
      if (k == 0 || kc5[k] >= KC5THRESHOLD) {
        syn[4 * l + 0] = S;
        syn[4 * l + 1] = syn[4 * l + 2] = syn[4 * l + 3] = 0.0;
      } else {
        const double dz = (k == nz - 1) ? 1e5 * std::fabs(c.Z(k) - c.Z(k - 1)) : 1e5 * std::fabs(c.Z(k + 1) - c.Z(k));
        double O[4][4];
        evol_operator(A, l, dz, O);
        double in[4] = {syn[4 * l], syn[4 * l + 1], syn[4 * l + 2], syn[4 * l + 3]};
        for (int i = 0; i < 4; ++i) {
          const double t1 = ((i == 0 ? 1.0 : 0.0) - O[i][0]) * S;
          const double t2 = O[i][0] * in[0] + O[i][1] * in[1] + O[i][2] * in[2] + O[i][3] * in[3];
          syn[4 * l + i] = t1 + t2;
        }
        for (int i = 0; i < 4; ++i)
          if (syn[4 * l + i] != syn[4 * l + i]) st = ORC_NAN;
      }
    }
  }
  // CALCULATE_EQUIVALENT_SYN1D: Stokes x GAIN, Stokes-major
  for (int i = 0; i < 4; ++i)
    for (int l = 0; l < numw; ++l) stokes[i * numw + l] = syn[4 * l + i] * (double)gain[4 * l + i];
  // log tau5, src/forward.f90:1000-1006
  std::vector<float> tau(nz);
  tau[nz - 1] = 1e-9f;
  for (int k = nz - 2; k >= 0; --k) {
    const float a = ((float)kc5[k] * c.RHO(k) + (float)kc5[k + 1] * c.RHO(k + 1)) / 2.0f;
    const double b = (c.Z(k + 1) - c.Z(k)) * 1000.0 * 100.0;
    tau[k] = (float)((double)tau[k + 1] + (double)a * b);
  }
  for (int k = 0; k < nz; ++k) c.TAU(k) = std::log10(tau[k]);
  return st;
}

#include "fz_oracle_rf.inc"

// ---------------------------------------------------- line database parse
// NCOLUMNS, src/lines_database.f90:145-190 (no commas in the database)
std::vector<std::string> split_ws(const std::string& ln) {
  std::vector<std::string> t;
  size_t i = 0;
  while (i < ln.size()) {
    while (i < ln.size() && (ln[i] == ' ' || ln[i] == '\t' || ln[i] == '\r')) ++i;
    size_t j = i;
    while (j < ln.size() && !(ln[j] == ' ' || ln[j] == '\t' || ln[j] == '\r')) ++j;
    if (j > i) t.push_back(ln.substr(i, j - i));
    i = j;
  }
  return t;
}

// ELECCONF, src/lines_database.f90:692-738
bool elecconf(const std::string& e, double& S, double& L, double& J) {
  if (e.size() < 7) return false;
  const float s = strtof(e.substr(0, 3).c_str(), nullptr);
  const float j = strtof(e.substr(4, 3).c_str(), nullptr);
  J = (double)j;
  S = ((double)s - 1.0) / 2.0;
  const char* ls = "SPDFGHI";
  const char* p = strchr(ls, e[3]);
  if (!p || !e[3]) return false;
  L = (double)(p - ls);
  return true;
}

// Numeric column of the 13-column format, src/lines_database.f90:245-270
double col13(const std::string& t) {
  double d;
  if (t.find('.') != std::string::npos) d = (double)strtof(t.c_str(), nullptr);
  else d = (double)(float)strtol(t.c_str(), nullptr, 10);
  return (double)std::llround(d * 1.0e6) * 1.0e-6;
}

// GET_NEFF, src/damping.f90:1016-1090
void get_neff(const orc_line& ln, bool lims, double& nlow, double& nupp) {
  double xlow = ln.eplow * EVOLT;
  double xupp = xlow + HPLA * LIGHT / (ln.l0 * sp(1e-8));
  double xh = fz_tab_xii[0] * EVOLT;
  double xll, xlu;
  if (lims) {
    xll = ln.elowlim;
    xlu = ln.eupplim;
  } else {
    double xlim = (ln.ion == 1 && ln.zn > 1) ? fz_tab_xi[ln.zn - 1] * EVOLT : fz_tab_xii[ln.zn - 1] * EVOLT;
    xll = xlim / (HPLA * LIGHT);
    xlu = xlim / (HPLA * LIGHT);
  }
  xlow = xlow / (HPLA * LIGHT);
  xupp = xupp / (HPLA * LIGHT);
  xh = xh / (HPLA * LIGHT);
  nlow = std::sqrt(xh / (xll - xlow));
  nupp = std::sqrt(xh / (xlu - xupp));
}

// TRANSITION_SP/PD/DF, src/damping.f90:1126-1305 (bilinear ABO look-up,
// including the grid-index quirk of TRANSITION_SP at :1160)
template <int NX, int NY>
void abo_interp(const double (*cs)[NY], const double (*al)[NY], double gx0, double gy0, double nx, double ny,
                bool quirk_sp, double& sigma, double& alpha) {
  double gx[NX], gy[NY];
  for (int i = 0; i < NX; ++i) gx[i] = gx0 + (double)i * sp(0.1);
  for (int i = 0; i < NY; ++i) gy[i] = gy0 + (double)i * sp(0.1);
  int ix = 0, iy = 0;
  for (int i = 1; i < NX; ++i)
    if (std::fabs(nx - gx[i]) < std::fabs(nx - gx[ix])) ix = i;
  for (int i = 1; i < NY; ++i)
    if (std::fabs(ny - gy[i]) < std::fabs(ny - gy[iy])) iy = i;
  if (nx < gx[ix]) ix -= 1;
  const double cmp = quirk_sp ? (sp(1.0) + (double)iy * sp(0.1)) : gy[iy];
  if (ny < cmp) iy -= 1;
  ix = std::max(0, std::min(ix, NX - 2));
  iy = std::max(0, std::min(iy, NY - 2));
  const double a1 = std::fabs((gx[ix + 1] - nx) * (gy[iy + 1] - ny));
  const double a2 = std::fabs((gx[ix] - nx) * (gy[iy + 1] - ny));
  const double a3 = std::fabs((gx[ix] - nx) * (gy[iy] - ny));
  const double a4 = std::fabs((gx[ix + 1] - nx) * (gy[iy] - ny));
  const double at = a1 + a2 + a3 + a4;
  sigma = (cs[ix][iy] * a1 + cs[ix + 1][iy] * a2 + cs[ix + 1][iy + 1] * a3 + cs[ix][iy + 1] * a4) / at;
  alpha = (al[ix][iy] * a1 + al[ix + 1][iy] * a2 + al[ix + 1][iy + 1] * a3 + al[ix][iy + 1] * a4) / at;
}

void collisional_param(orc_line& ln, double nlow, double nupp) {
  const int tt = ln.otr[0] + ln.otr[1];
  int ierr = 0;
  double sig = ln.sigma, alp = ln.alpha;
  if (tt == 1) {
    double nss = 0, nsp = 0;
    if (ln.otr[0] == 0) nss = nlow;
    if (ln.otr[0] == 1) nsp = nlow;
    if (ln.otr[1] == 0) nss = nupp;
    if (ln.otr[1] == 1) nsp = nupp;
    if (nss > 5.5 || nss < 1. || nsp > 5.5 || nsp < sp(1.3)) ierr = 3;
    if (!ierr) abo_interp<46, 43>(fz_tab_abo_cs_sp, fz_tab_abo_al_sp, 1.0, sp(1.3), nss, nsp, true, sig, alp);
  } else if (tt == 3) {
    double nsp = 0, nsd = 0;
    if (ln.otr[0] == 1) nsp = nlow;
    if (ln.otr[0] == 2) nsd = nlow;
    if (ln.otr[1] == 1) nsp = nupp;
    if (ln.otr[1] == 2) nsd = nupp;
    if (nsp > 5.5 || nsp < sp(1.3) || nsd > 5.5 || nsd < sp(2.3)) ierr = 3;
    if (!ierr) abo_interp<43, 33>(fz_tab_abo_cs_pd, fz_tab_abo_al_pd, sp(1.3), sp(2.3), nsp, nsd, false, sig, alp);
  } else if (tt == 5) {
    double nsd = 0, nsf = 0;
    if (ln.otr[0] == 2) nsd = nlow;
    if (ln.otr[0] == 3) nsf = nlow;
    if (ln.otr[1] == 2) nsd = nupp;
    if (ln.otr[1] == 3) nsf = nupp;
    if (nsd > 5.5 || nsd < sp(2.3) || nsf > 6. || nsf < sp(3.3)) ierr = 3;
    if (!ierr) abo_interp<33, 28>(fz_tab_abo_cs_df, fz_tab_abo_al_df, sp(2.3), sp(3.3), nsd, nsf, false, sig, alp);
  } else {
    ierr = 1;
  }
  ln.abo_ierr = ierr;
  if (!ierr) {
    ln.sigma = sig;
    ln.alpha = alp;
  }
}

}  // namespace

// =========================================================== C entry points
extern "C" {

int orc_version(void) { return 1; }

// Test hook: replace the abundance set (NULL restores ATOM_INIT's Thevenin
// 1989 values).  Not thread safe; call before any computation.
void orc_set_abundances(const double* abund92) { set_abund(abund92); }

void orc_partition(int zn, double T, double out6[6]) {
  double U[3], dU[3];
  partition(zn, T, U, dU);
  for (int i = 0; i < 3; ++i) {
    out6[i] = U[i];
    out6[3 + i] = dU[i];
  }
}

int orc_get_rho(double T, double pg, double* nelec, double out5[5]) {
  Rho r = get_rho(T, pg, *nelec);
  out5[0] = r.nhyd;
  out5[1] = r.pelec;
  out5[2] = r.dens;
  out5[3] = r.molecw;
  out5[4] = r.iters;
  return r.status;
}

double orc_opac_continuum(float T, double lambda0, double ne, double nh) { return opac_continuum(T, lambda0, ne, nh); }

int orc_parse_lines(const char* text, orc_line* out, int maxn) {
  std::string all(text);
  size_t pos = 0;
  int n = 0;
  std::string shell = "  ";
  bool ended = false;
  while (pos < all.size()) {
    size_t e = all.find('\n', pos);
    if (e == std::string::npos) e = all.size();
    std::string ln = all.substr(pos, e - pos);
    pos = e + 1;
    std::vector<std::string> t = split_ws(ln);
    if (t.empty()) continue;
    if (t.size() == 1 && t[0] == "END") {
      ended = true;
      break;
    }
    if (n >= maxn) return -2;
    orc_line L{};
    if (t.size() == 13) {
      L.num = (int)strtol(t[0].c_str(), nullptr, 10);
      L.zn = (int)strtol(t[1].c_str(), nullptr, 10);
      L.ion = (int)strtol(t[2].c_str(), nullptr, 10);
      L.l0 = col13(t[3]);
      if (!elecconf(t[4], L.sl, L.ll, L.jl) || !elecconf(t[5], L.su, L.lu, L.ju)) return -3;
      L.loggf = col13(t[6]);
      L.eplow = col13(t[7]);
      L.alpha = col13(t[8]);
      L.sigma = col13(t[9]);
      shell = t[10].substr(0, 2);
      L.elowlim = col13(t[11]);
      L.eupplim = col13(t[12]);
    } else if (t.size() == 8) {
      L.num = (int)strtol(t[0].c_str(), nullptr, 10);
      L.zn = (int)strtol(t[1].c_str(), nullptr, 10);
      L.ion = (int)strtol(t[2].c_str(), nullptr, 10);
      auto c8 = [](const std::string& s) { return (double)std::lround(strtod(s.c_str(), nullptr) * 1.e4) * 1.e-4; };
      L.l0 = c8(t[3]);
      if (!elecconf(t[4], L.sl, L.ll, L.jl) || !elecconf(t[5], L.su, L.lu, L.ju)) return -3;
      L.loggf = c8(t[6]);
      L.eplow = c8(t[7]);
    } else {
      return -4;
    }
    // OPTICAL_ELEC_TRAN, src/lines_database.f90:742-787
    L.flag = 1;
    for (int i = 0; i < 2; ++i) {
      const char ch = i < (int)shell.size() ? shell[i] : ' ';
      L.flag = 1;
      switch (ch) {
        case 's': case 'S': L.otr[i] = 0; L.flag = 0; break;
        case 'p': case 'P': L.otr[i] = 1; L.flag = 0; break;
        case 'd': case 'D': L.otr[i] = 2; L.flag = 0; break;
        case 'f': case 'F': L.otr[i] = 3; L.flag = 0; break;
        default: break;
      }
    }
    L.abo_ierr = -1;
    if ((L.alpha == 0.0 || L.sigma == 0.0) && L.flag == 0) {
      double nlow, nupp;
      const bool lims = (L.elowlim != 0.0 && L.eupplim != 0.0);
      get_neff(L, lims, nlow, nupp);
      collisional_param(L, nlow, nupp);
    }
    out[n++] = L;
  }
  return ended ? n : -1;
}

int orc_zeeman(const orc_line* ln, double* shift, double* strength, int* type, int maxn) {
  Zeeman z = zeeman(*ln);
  for (int i = 0; i < z.n && i < maxn; ++i) {
    shift[i] = z.shift[i];
    strength[i] = z.strength[i];
    type[i] = z.type[i];
  }
  return z.n;
}

void orc_voigt(int n, double a, const double* v, double* h, double* f) {
  for (int i = 0; i < n; ++i) voigt1(a, v[i], h[i], f[i]);
}

// SET_BOUNDARY + OLD_ANALYTICAL_SOLVER (src/rtesolver.f90:163-187,
// :1134-1147) on given absorption-matrix elements and source functions:
// from the bottom up, I = (S, 0, 0, 0) at K = 1 and wherever bnd[K] is set,
// else I_K = (1 - O_K) S_K + O_K I_{K-1}, O_K = EVOL_OPERATOR of the
// height's matrix over dz = 1e5 |z_{K+1} - z_K| cm (the top height's
// backward difference).  eta: (7, nw, nz) as ETAI, ETAQ, ETAU, ETAV, RHOQ,
// RHOU, RHOV (nw fastest); src (nw, nz); out (4, nw) SYN1D.
void orc_rte_solve(int nz, int nw, const double* eta, const double* src, const double* zz, const int* bnd,
                   double* out) {
  AbsMat A;
  A.resize(nw);
  std::vector<double*> rows = {A.ei.data(), A.eq.data(), A.eu.data(), A.ev.data(), A.rq.data(), A.ru.data(),
                               A.rv.data()};
  for (int k = 0; k < nz; ++k) {
    for (int e = 0; e < 7; ++e)
      for (int l = 0; l < nw; ++l) rows[e][l] = eta[((size_t)k * 7 + e) * nw + l];
    for (int l = 0; l < nw; ++l) {
      const double S = src[(size_t)k * nw + l];
      double* o = out + 4 * (size_t)l;
      if (k == 0 || (bnd && bnd[k])) {
        o[0] = S;
        o[1] = o[2] = o[3] = 0.0;
        continue;
      }
      const double dz = (k == nz - 1) ? 1e5 * std::fabs(zz[k] - zz[k - 1]) : 1e5 * std::fabs(zz[k + 1] - zz[k]);
      double O[4][4];
      evol_operator(A, l, dz, O);
      const double in[4] = {o[0], o[1], o[2], o[3]};
      for (int i = 0; i < 4; ++i)
        o[i] = ((i == 0 ? 1.0 : 0.0) - O[i][0]) * S + O[i][0] * in[0] + O[i][1] * in[1] + O[i][2] * in[2] +
               O[i][3] * in[3];
    }
  }
}

// GET_NORM, src/normalization.f90:696-754
int orc_gain(const orc_line* lines, int nlines, const orc_region* regs, int nreg, float* gain) {
  Setup s = make_setup(lines, nlines, regs, nreg);
  const int numw = s.numw, N = FZ_HSRA_LEN;
  std::vector<double> syn(numw, 0.0), kc(nreg);
  double nelec = 0.0;
  int st = 0;
  for (int k = 0; k < N; ++k) {
    const float T = fz_tab_hsra_tem[k];
    Rho r = get_rho((double)T, (double)fz_tab_hsra_pg[k], nelec);
    if (r.status) st = r.status;
    for (int L = 0; L < nreg; ++L) kc[L] = opac_continuum(T, s.lines[s.regs[L].line[0]].l0, nelec, r.nhyd);
    for (int l = 0; l < numw; ++l) {
      const int L = s.regof[l];
      double w = s.lines[s.regs[L].line[0]].l0 + s.wave[l] / 1e3;
      w = w * 1e-8;
      const double S = (double)(float)(2.0 * HPLA * std::pow(LIGHT, 2.0) / std::pow(w, 5.0) *
                                       (1.0 / (std::exp(HPLA * LIGHT / (w * KBOL * (double)T)) - 1.0)));
      if (k == 0) {
        syn[l] = S;
      } else {
        double ei = kc[L];
        const bool imat = (ei == ei + 1.0);
        if (imat) ei = 1e15;
        const double dz = (k == N - 1) ? 1e5 * (double)std::fabs(fz_tab_hsra_z[k] - fz_tab_hsra_z[k - 1])
                                       : 1e5 * (double)std::fabs(fz_tab_hsra_z[k + 1] - fz_tab_hsra_z[k]);
        double ev = std::exp(-ei * dz) * (0.5 * (1.0 + 1.0) * 1.0);
        if (imat) ev = 1.0;
        syn[l] = (double)(float)((1.0 - ev) * S + ev * syn[l]);
      }
    }
  }
  for (int l = 0; l < numw; ++l) {
    const float g = (float)(1.0 / syn[l]);
    gain[4 * l + 0] = g;
    gain[4 * l + 1] = g;
    gain[4 * l + 2] = g;
    gain[4 * l + 3] = -g;
  }
  return st;
}

int orc_forward(const orc_line* lines, int nlines, const orc_region* regs, int nreg, const float* gain, int nz,
                int ncol, float* model, int hydrostatic, double* stokes, int* status, int nthreads) {
  Setup s = make_setup(lines, nlines, regs, nreg);
  const int numw = s.numw;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int i = 0; i < ncol; ++i) {
    Col c{model + (size_t)i * nz * 13, nz};
    status[i] = forward1d(s, gain, c, hydrostatic, stokes + (size_t)i * 4 * numw);
  }
  (void)nthreads;
  return 0;
}

int orc_forward_rf(const orc_line* lines, int nlines, const orc_region* regs, int nreg, const float* gain, int nz,
                   int ncol, float* model, int hydrostatic, const int* nodes, double* stokes, float* jac, int* status,
                   int nthreads) {
  int np = 0;
  for (int p = 1; p <= 8; ++p) {
    if (nodes[p - 1] <= 0) continue;
    if (p == 3 || p == 8) return -1;   // constant-density pair and P0 are not restated
    if (nodes[p - 1] > nz) return -2;   // GET_INT_COEFS stops when NJ > NZ
    np += nodes[p - 1];
  }
  Setup s = make_setup(lines, nlines, regs, nreg);
  const int numw = s.numw;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int i = 0; i < ncol; ++i) {
    Col c{model + (size_t)i * nz * 13, nz};
    status[i] = forward1d_rf(s, gain, c, hydrostatic, nodes, stokes + (size_t)i * 4 * numw,
                             jac + (size_t)i * 4 * numw * np);
  }
  (void)nthreads;
  return np;
}

}  // extern "C"
