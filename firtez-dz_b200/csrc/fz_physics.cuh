// Device physics of the Stokes synthesis path (sm_100a).
//
//  * FP64, one warp per column, lanes over the 92 elements: partition
//    functions, Saha ionisation equilibrium and the damped electron-density
//    fixed point GET_RHO (src/chemical_equilibrium.f90:165-278, :1601-1701),
//    continuum opacity (src/cont_opacity.f90:48-357), line opacity
//    (src/line_opacity.f90:34-108) and damping (src/damping.f90:842-1012).
//  * FP32, one thread per wavelength: Hui-Armstrong-Wray Voigt/Faraday
//    (src/voigt.f:17-98) and the Landi Degl'Innocenti evolution operator
//    (src/rtesolver.f90:269-473) written on per-layer optical depths.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define FZ_TABLE_QUAL static __device__ const
#include "fz_tables.h"

namespace fzd {

// ------------------------------------------------------------------ constants
struct Consts {
  double csaha1, csaha2, rbohr, deno_sa, deno_sam;
  double ab10[FZ_NELEM];   // 10**(ABUND-12)
};

constexpr double DPI = 3.141592653589793238462643;
constexpr double LIGHT = 2.99792458e+10;
constexpr double KBOL = 1.38056503e-16;
constexpr double MELE = 9.10938215e-28;
constexpr double QELE = 4.80320425e-10;
constexpr double EVOLT = 1.60217656e-12;
constexpr double MAMU = 1.66053892e-24;
constexpr double HPLA = 6.62606957e-27;
constexpr double GRAV = 2.7414e4;
constexpr double KC5THRESHOLD = 2.0e10;   // src/forward.f90:884

__device__ __forceinline__ double spd(float x) { return (double)x; }

// ------------------------------------------------------- partition functions
__device__ __forceinline__ double horner_exact(const double* c, int n, double x) {
  double r = c[n - 1];
  for (int i = n - 2; i >= 0; --i) r = __dadd_rn(c[i], __dmul_rn(x, r));
  return r;
}

__device__ __forceinline__ bool pf_cond(int cond, double th, double T, double u) {
  return cond == 0 || (cond == 1 && T > th) || (cond == 2 && T < th) || (cond == 3 && T <= th) ||
         (cond == 4 && T >= th) || (cond == 5 && u != th);
}

__device__ __forceinline__ double pf_vpiece(const fz_pf_vpiece& p, const double var[3]) {
  const double h = horner_exact(p.c, p.nc, var[p.var]);
  if (p.form == 1) return p.base + exp(h);
  if (p.form == 2) return fmax(p.clamp, h);
  return h;
}

// U_I, U_II, U_III of element zn (1-based), src/atom_database.f90:121-1035.
__device__ __forceinline__ void partition_u(int zn, double T, const double var[3], double U[3]) {
  const int e = zn - 1;
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int nv = fz_tab_pf_nv[e][s];
    int act = -1;
    for (int i = 0; i < nv; ++i)
      if (pf_cond(fz_tab_pf_v[e][s][i].cond, fz_tab_pf_v[e][s][i].th, T, 0.0)) act = i;
    U[s] = act >= 0 ? pf_vpiece(fz_tab_pf_v[e][s][act], var) : 0.0;
  }
}

// --------------------------------------------------------- warp chemistry
// Per-lane Saha factors of elements lane, lane+32, lane+64 at temperature T
// (SHORT_PRE_ION_CALC_TEMPRHO, src/chemical_equilibrium.f90:1601-1652).
struct WarpSaha {
  double T;
  double a1[3], a2[3];
};

__device__ __forceinline__ double clamp650(double e) {
  if (e > 0.0) e = fmin(e, 650.0);
  if (e < 0.0) e = fmax(e, -650.0);
  return e;
}

__device__ void saha_prepare(WarpSaha& w, double T, const Consts& K, int lane) {
  w.T = T;
  const double lamelec = K.csaha1 * pow(T, -3.0 / 2.0);
  const double var[3] = {T, 1.0e-3 * T, log(5040.0 / T)};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int e = lane + 32 * j;
    w.a1[j] = 0.0;
    w.a2[j] = 0.0;
    if (e < FZ_NELEM) {
      double U[3];
      partition_u(e + 1, T, var, U);
      const double e1 = exp(clamp650(K.csaha2 * fz_tab_xi[e] / T));
      const double e2 = exp(clamp650(K.csaha2 * fz_tab_xii[e] / T));
      w.a1[j] = (U[0] / (2.0 * U[1])) * lamelec * e1;
      w.a2[j] = (U[1] / (2.0 * U[2])) * lamelec * e2;
    }
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;   // xor butterfly: bit-identical in every lane
}

struct RhoOut {
  double nhyd, pelec, dens, molecw;
  int status;
};

// GET_RHO, src/chemical_equilibrium.f90:165-278.  All lanes of the warp call
// it with the same arguments; nelec (the warm-start chain) is updated in
// every lane identically.
__device__ RhoOut get_rho_warp(const WarpSaha& w, double PG, double& nelec, const Consts& K, int lane) {
  RhoOut r;
  const double T = w.T;
  double nhyd = 0.0;
  if (nelec != nelec) nelec = 0.0;
  if (nelec < 1.0) nelec = PG / (101.0 * KBOL * T);
  const double pelec = nelec * KBOL * T;
  if (pelec > PG) nelec = (PG * 0.5) / (KBOL * T);
  double err = 1.0;
  int iter = 1;
  double nnew = nelec, nold = nelec;
  while (err > 1.0e-4 && iter <= 100 && nhyd >= 0.0) {
    nold = nnew;
    const double nume = PG - nnew * KBOL * T;
    nhyd = nume / (K.deno_sa * KBOL * T);
    const double ne = nnew;
    double h = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int e = lane + 32 * j;
      if (e < FZ_NELEM) {
        const double vnt = nhyd * K.ab10[e];
        const double na1 = ne * w.a1[j], na2 = ne * w.a2[j];
        const double r2 = 1.0 / na2;
        const double vnii = vnt / (na1 + 1.0 + r2);
        const double vniii = vnt / (1.0 + na2 * (na1 + 1.0));
        if (e == 0) {
          const double vni = vnt / (1.0 + (1.0 / na1) * (1.0 + r2));
          h = vniii - vni;
        } else {
          s2 += vnii;
          s3 += vniii;
        }
      }
    }
    h = warp_sum(h);
    s2 = warp_sum(s2);
    s3 = warp_sum(s3);
    double est = h;
    est = est + s2 + s3;
    nnew = (fmax(est, 0.0) + nold) / 2.0;
    err = fabs((nnew - nold) / nnew);
    iter = iter + 1;
  }
  r.status = 0;
  if (iter >= 100 || nhyd < 0.0) r.status = 1;
  nelec = nnew;
  const double nume = PG - nelec * KBOL * T;
  nhyd = nume / (K.deno_sa * KBOL * T);
  r.dens = nhyd * K.deno_sam + nelec * MELE;
  r.molecw = ((r.dens * KBOL * T) / MAMU) * (1.0 / PG);
  if (nhyd != nhyd || nnew != nnew) r.status = 2;
  if (nelec < 0.0 || nhyd <= 0.0) r.status = 1;
  r.nhyd = nhyd;
  r.pelec = pelec;   // pressure of the initial guess, as the reference returns it
  return r;
}

// ----------------------------------------------------- continuum opacity
__device__ double hminus_ff(double T, double ne, double l0) {
  const double A1[6] = {0, 2483.346, -3449.889, 2200.04, -696.271, 88.283};
  const double B1[6] = {0, 285.827, -1158.382, 2427.719, -1841.4, 444.517};
  const double C1[6] = {0, -2054.291, 8746.523, -13651.105, 8624.97, -1863.864};
  const double D1[6] = {0, 2827.776, -11485.632, 16755.524, -10051.53, 2095.288};
  const double E1[6] = {0, -1341.537, 5303.609, -7510.494, 4400.067, -901.788};
  const double F1[6] = {0, 208.952, -812.939, 1132.738, -655.02, 132.985};
  const double A2[4] = {518.1021, 473.2636, -482.2089, 115.5291};
  const double B2[4] = {-734.8666, 1443.4137, -737.1616, 169.6374};
  const double C2[4] = {1021.1775, -1977.3395, 1096.8827, -245.649};
  const double D2[4] = {-479.0721, 922.3575, -521.1341, 114.243};
  const double E2[4] = {93.1373, -178.9275, 101.7963, -21.9972};
  const double F2[4] = {-6.4285, 12.36, -7.0571, 1.5097};
  const double lm = l0 / 1e4;
  const double th = 5040.0 / T;
  const double lm2 = pow(lm, 2.0), lm3 = pow(lm, 3.0), lm4 = pow(lm, 4.0);
  double part1;
  if (lm < 0.3645) {
    double c[4];
    for (int i = 0; i < 4; ++i) c[i] = A2[i] * lm2 + B2[i] + C2[i] / lm + D2[i] / lm2 + E2[i] / lm3 + F2[i] / lm4;
    part1 = c[0] * th + c[1] * pow(th, 1.5) + c[2] * pow(th, 2.0) + c[3] * pow(th, 2.5);
  } else {
    double c[6];
    for (int i = 0; i < 6; ++i) c[i] = A1[i] * lm2 + B1[i] + C1[i] / lm + D1[i] / lm2 + E1[i] / lm3 + F1[i] / lm4;
    part1 = c[0] * th + c[1] * pow(th, 1.5) + c[2] * pow(th, 2.0) + c[3] * pow(th, 2.5) + c[4] * pow(th, 3.0) +
            c[5] * pow(th, 3.5);
  }
  return 1e-29 * part1 * KBOL * ne * T;
}

__device__ double hminus_bf(double T, double ne, double l0) {
  const double LAMBDAP = 1.6419, CTE = 0.75e-18;
  const double ALPHA = (HPLA * LIGHT / KBOL) * 1e4;
  const double CC[6] = {152.519, 49.534, -118.858, 92.536, -34.194, 4.982};
  const double lm = l0 / 1e4;
  if (!(lm < LAMBDAP)) return 0.0;
  const double com = 1.0 / lm - 1.0 / LAMBDAP;
  double sigma = CC[0] + CC[1] * pow(com, 0.5) + CC[2] * com + CC[3] * pow(com, 1.5) + CC[4] * pow(com, 2.0) +
                 CC[5] * pow(com, 2.5);
  sigma = CTE * sigma * pow(lm, 3.0) * pow(com, 1.5);
  const double part = pow(T, -2.5) * exp(ALPHA / (T * LAMBDAP)) * (1.0 - exp(-ALPHA / (T * lm)));
  return part * sigma * ne * KBOL * T;
}

__device__ double opac_continuum(float Tsp, double l0, double ne, double nh) {
  const double T = (double)Tsp;
  // THOMSON, :187-217
  const double CT = (8.0 * DPI / 3.0) * (pow(QELE / LIGHT, 4.0)) / pow(MELE, 2.0);
  const double thom = CT * (ne / nh);
  // RAYLEIGH_H, :221-239
  const double ray = (5.799e-13 + (1.422e-6 + 2.784 / pow(l0, 2.0)) / pow(l0, 2.0)) / pow(l0, 4.0);
  // HYDROGEN, :243-301 (REAL*4 literals 13.595 and 1E-8)
  const double IOPOT = (double)13.595f;
  const double E8 = (double)1e-8f;
  const double C1 = E8 * IOPOT * EVOLT / (HPLA * LIGHT);
  const double C2 = pow(E8, 3.0) * 64.0 * pow(DPI, 4.0) * MELE * pow(QELE, 10.0) /
                    (3.0 * sqrt(3.0) * pow(LIGHT, 4.0) * pow(HPLA, 6.0));
  const double C3 = HPLA * LIGHT / (KBOL * E8);
  const double C4 = IOPOT * EVOLT / KBOL;
  const int n0 = 1 + (int)floor(sqrt(C1 * l0));
  double sum;
  if (n0 <= 8) {
    sum = exp(C4 / (T * pow((double)n0, 2.0))) * pow((double)n0, -3.0);
    for (int i = n0 + 1; i <= 8; ++i) sum = sum + exp(C4 / (T * pow((double)i, 2.0))) * pow((double)i, -3.0);
    sum = sum + (0.117 + exp(C4 / (T * pow(9.0, 2.0)))) * (T / (2.0 * C4));
  } else {
    sum = (0.117 + exp(C4 / (T * pow((double)n0, 2.0)))) * (T / (2.0 * C4));
  }
  const double hyd = C2 * sum * (1.0 - exp(-C3 / (T * l0))) * exp(-C4 / T) * pow(l0, 3.0);
  const double factor = hminus_ff(T, ne, l0) + hminus_bf(T, ne, l0) + thom + ray + hyd;
  return nh * factor;
}

// ------------------------------------------------------ line opacity, damping
struct LineP {   // one spectral line, FP64 constants
  double l0, loggf, eplow, alpha, sigma, matom, abund, wdif;
  int zn, ion;
};

// ION_CALC_TEMPX (value), src/chemical_equilibrium.f90:1511-1597
__device__ double ion_calc_tempx(int zn, int ion, double T, double ne, double n, const Consts& K, double* upi) {
  const double var[3] = {T, 1.0e-3 * T, log(5040.0 / T)};
  double U[3];
  partition_u(zn, T, var, U);
  const double lamelec = K.csaha1 * pow(T, -3.0 / 2.0);
  const double e1 = exp(clamp650(K.csaha2 * fz_tab_xi[zn - 1] / T));
  const double e2 = exp(clamp650(K.csaha2 * fz_tab_xii[zn - 1] / T));
  const double al1 = (U[0] / (2.0 * U[1])) * lamelec * e1;
  const double al2 = (U[1] / (2.0 * U[2])) * lamelec * e2;
  const double deno = pow(ne, 2.0) * al1 * al2 + ne * al2 + 1.0;
  double nume = 1.0;
  if (ion == 1) nume = pow(ne, 2.0) * al1 * al2;
  if (ion == 2) nume = ne * al2;
  *upi = U[ion - 1];
  return n * nume / deno;
}

// OPAC_LINE, src/line_opacity.f90:34-108 (LTE)
__device__ double opac_line(const LineP& L, float Tsp, double ne, double nh, const Consts& K) {
  const double T = (double)Tsp;
  const double n = nh * pow(10.0, L.abund - 12.0);
  double upi;
  const double npi = ion_calc_tempx(L.zn, L.ion, T, ne, n, K, &upi);
  const double t1 = sqrt(DPI) * pow(QELE, 2.0) / (MELE * LIGHT) * pow(10.0, L.loggf) * L.l0 * 1e-8;
  const double t2 = sqrt(L.matom * MAMU / (2.0 * KBOL * T));
  const double t3 = 1.0 * npi / upi;
  const double t4 = exp(-L.eplow * EVOLT / (KBOL * T));
  const double t5 = 1.0 - (1.0 / 1.0) * exp(-HPLA * LIGHT / (1.0e-8 * L.l0 * KBOL * T));
  return t1 * t2 * t3 * t4 * t5;
}

// REFRAX, src/atom_database.f90:1039-1074
__device__ double refrax(double w) {
  const double T = 15.0, P = 760.0, H = 0.0;
  const double s = 1.0 / pow(w, 2.0);
  const double r = 6.4328e-5 + 2.94981e-2 / (146.0 - s) + 2.554e-4 / (41.0 - s);
  const double y = 1.0 / (273.15 + T);
  const double alpha = 3.67e-3 + 3.3e-4 * exp((0.19 - w) / 0.12);
  const double wvsp =
      pow(10.0, -55.1132754 +
                    y * (1.19551822e5 +
                         y * (-9.70108858e7 + y * (4.12856913e10 + y * (-9.87931835e12 + y * (1.25868645e15 - 6.66885272e16 * y))))));
  const double wvp = 1.0e-2 * H * wvsp;
  return 1.0 + 1.31579e-3 * r * P / (1.0 + alpha * (T - 1.0) / (1.0 + 15.0 * alpha)) - 5.49e-8 * wvp / (1.0 + alpha * T);
}

// GET_DAMPING, src/damping.f90:842-1012 (value)
__device__ double get_damping(const LineP& L, double nhyd, float Tsp, const Consts& K, double matom_h,
                              double matom_he, double abund_he) {
  const double lambda = L.l0 * 1e-8;
  const double T8 = (double)Tsp;
  const double RAT = (double)0.3181818f;
  const double m = L.matom;
  const double vdop = sqrt(2.0 * KBOL * T8 / (MAMU * m));
  const double grad = 0.2223 / pow(lambda, 2.0);
  const double mu_h = MAMU * (m * matom_h) / (m + matom_h);
  const double mu_he = MAMU * (m * matom_he) / (m + matom_he);
  const double nhe = nhyd * pow(10.0, abund_he - 12.0);
  double gcol;
  if (L.sigma > 0 && L.alpha > 0) {
    const double e1 = 2.0 - L.alpha / 2.0;
    const double e2 = (1.0 - L.alpha) / 2.0;
    const double gammaf =
        1.0 + (-0.5748646 + (0.9512363 + (-0.6998588 + (0.4245549 - 0.1010678 * e1) * e1) * e1) * e1) * e1;
    double beta = pow(4.0 / DPI, L.alpha / 2.0) * gammaf * pow(1e6, L.alpha) * (L.sigma * pow(K.rbohr, 2.0)) *
                  pow(8.0 * KBOL / DPI, e2);
    beta = 2.0 * beta;
    gcol = beta * pow(T8, e2) * (nhyd * pow(mu_h, -e2) + RAT * nhe * pow(mu_he, -e2));
  } else {
    double rindex = (double)1.0004f;
    if (lambda * 1e8 >= 1800.0) rindex = refrax(lambda * 1e4);
    const double lvac = rindex * lambda;
    const double epupp = L.eplow + (HPLA * LIGHT / lvac) / EVOLT;
    const double xi = fz_tab_xi[L.zn - 1], xii = fz_tab_xii[L.zn - 1];
    const double ionf = (double)(float)(L.ion - 1);
    double ed1, ed2, chyd;
    if (L.ion == 1) {
      ed1 = fmax(xi - epupp - xi * ionf, 1.0);
      ed2 = fmax(xi - L.eplow - xi * ionf, 3.0);
      chyd = 1.0;
    } else {
      ed1 = fmax(xii - epupp - xi * ionf, 1.0);
      ed2 = fmax(xii - L.eplow - xi * ionf, 3.0);
      chyd = (double)1.741f;
    }
    chyd = chyd * 17.0 * pow(8.0 * KBOL / DPI, 0.3);
    chyd = chyd * pow(pow(10.0, -30.5325) * (1.0 / pow(ed1, 2.0) - 1.0 / pow(ed2, 2.0)), 0.4);
    const double chydp = chyd * (nhyd * pow(mu_h, -0.3) + nhe * pow(mu_he, -0.3));
    gcol = chydp * pow(T8, 0.3);
  }
  return (grad + gcol) * lambda / (4.0 * DPI * vdop);
}

// ------------------------------------------------------------ FP32 Voigt
// Hui, Armstrong & Wray (1978) 7-pole rational approximation of the complex
// probability function, as src/voigt.f:17-98: H = Re w, F = sign(v) Im w
// with w evaluated at z = a - i|v|.  Division by range reduction (Smith).
__device__ __forceinline__ void voigt_f32(float a, float u, float& H, float& F) {
  const float A0 = 122.607931777104326f, A1 = 214.382388694706425f, A2 = 181.928533092181549f,
              A3 = 93.155580458138441f, A4 = 30.180142196210589f, A5 = 5.912626209773153f,
              A6 = .564189583562615f, B0 = 122.60793177387535f, B1 = 352.730625110963558f,
              B2 = 457.334478783897737f, B3 = 348.703917719495792f, B4 = 170.354001821091472f,
              B5 = 53.992906912940207f, B6 = 10.479857114260399f;
  const float v = fabsf(u);
  const float zr = a, zi = -v;
  // numerator
  float nr = fmaf(A6, zr, A5), ni = A6 * zi;
  float tr, ti;
#define FZ_CSTEP(C)                        \
  tr = fmaf(nr, zr, -ni * zi) + (C);       \
  ti = fmaf(nr, zi, ni * zr);              \
  nr = tr;                                 \
  ni = ti;
  FZ_CSTEP(A4) FZ_CSTEP(A3) FZ_CSTEP(A2) FZ_CSTEP(A1) FZ_CSTEP(A0)
  float dr = zr + B6, di = zi;
#define FZ_DSTEP(C)                        \
  tr = fmaf(dr, zr, -di * zi) + (C);       \
  ti = fmaf(dr, zi, di * zr);              \
  dr = tr;                                 \
  di = ti;
  FZ_DSTEP(B5) FZ_DSTEP(B4) FZ_DSTEP(B3) FZ_DSTEP(B2) FZ_DSTEP(B1) FZ_DSTEP(B0)
#undef FZ_CSTEP
#undef FZ_DSTEP
  float wr, wi;
  if (fabsf(dr) >= fabsf(di)) {
    const float r = __fdividef(di, dr);
    const float den = __frcp_rn(fmaf(di, r, dr));
    wr = fmaf(ni, r, nr) * den;
    wi = fmaf(-nr, r, ni) * den;
  } else {
    const float r = __fdividef(dr, di);
    const float den = __frcp_rn(fmaf(dr, r, di));
    wr = fmaf(nr, r, ni) * den;
    wi = fmaf(ni, r, -nr) * den;
  }
  H = wr;
  F = (u < 0.0f) ? -wi : wi;
}

// Evolution operator O of one layer from its optical-depth increments
// t = eta*dz (src/rtesolver.f90:269-473).  The reference's clamp of cosh and
// sinh at 2^53 (-> 1e15, :464-465) is reproduced; below it the operator is
// evaluated with cancellation-free forms (cosh x -+ cos y via sinh^2(x/2),
// sin^2(y/2); lambda_1,2 from the larger root).
__device__ __forceinline__ void evol_f32(float tI, float tQ, float tU, float tV, float rQ, float rU, float rV,
                                         float O[16]) {
  const float eta2 = tQ * tQ + tU * tU + tV * tV;
  const float rho2 = rQ * rQ + rU * rU + rV * rV;
  const float er = tQ * rQ + tU * rU + tV * rV;
  const float d = eta2 - rho2;
  const float R = sqrtf(0.25f * d * d + er * er);
  float x, y;   // lambda_1 dz, lambda_2 dz
  if (d >= 0.0f) {
    x = sqrtf(R + 0.5f * d);
    y = x > 0.0f ? fabsf(er) / x : 0.0f;
  } else {
    y = sqrtf(R - 0.5f * d);
    x = y > 0.0f ? fabsf(er) / y : 0.0f;
  }
  const float sg = er > 0.0f ? 1.0f : (er < 0.0f ? -1.0f : 0.0f);
  const float theta = 2.0f * R;
  const float it = theta > 0.0f ? 1.0f / theta : 0.0f;
  // M2, M3, M4 (Fortran (row,col) -> O[4*(row-1)+(col-1)])
  const float m2_21 = (y * tQ - sg * x * rQ) * it, m2_31 = (y * tU - sg * x * rU) * it,
              m2_41 = (y * tV - sg * x * rV) * it;
  const float m2_32 = (sg * x * tV + y * rV) * it, m2_42 = (-sg * x * tU - y * rU) * it,
              m2_43 = (sg * x * tQ + y * rQ) * it;
  const float m3_21 = (x * tQ + sg * y * rQ) * it, m3_31 = (x * tU + sg * y * rU) * it,
              m3_41 = (x * tV + sg * y * rV) * it;
  const float m3_32 = (-sg * y * tV + x * rV) * it, m3_42 = (sg * y * tU - x * rU) * it,
              m3_43 = (-sg * y * tQ + x * rQ) * it;
  const float m4_11 = (eta2 + rho2) * it;   // 2*((eta2+rho2)/2)/theta
  const float m4_21 = 2.0f * (tV * rU - tU * rV) * it, m4_31 = 2.0f * (tQ * rV - tV * rQ) * it,
              m4_41 = 2.0f * (tU * rQ - tQ * rU) * it;
  const float m4_22 = 2.0f * (tQ * tQ + rQ * rQ) * it - m4_11, m4_33 = 2.0f * (tU * tU + rU * rU) * it - m4_11,
              m4_44 = 2.0f * (tV * tV + rV * rV) * it - m4_11;
  const float m4_32 = 2.0f * (tQ * tU + rQ * rU) * it, m4_42 = 2.0f * (tV * tQ + rV * rQ) * it,
              m4_43 = 2.0f * (tU * tV + rU * rV) * it;
  const float E = expf(-tI);
  float P, Qm, sh, s2v;
  const float XCLAMP = 37.42994775f;   // cosh, sinh >= 2^53 in float64
  s2v = sinf(y);
  if (x >= XCLAMP) {
    const float c2 = cosf(y);
    P = 0.5f * (1e15f + c2);
    Qm = 0.5f * (1e15f - c2);
    sh = 1e15f;
  } else {
    const float shx = sinhf(0.5f * x), siy = sinf(0.5f * y);
    const float a = shx * shx, b = siy * siy;
    P = 1.0f + a - b;
    Qm = a + b;
    sh = sinhf(x);
  }
  const float eP = E * P, eQ = E * Qm, eS = E * s2v, eH = E * sh;
  O[0] = eP + eQ * m4_11;
  O[5] = eP + eQ * m4_22;
  O[10] = eP + eQ * m4_33;
  O[15] = eP + eQ * m4_44;
  // (2,1),(1,2): M2,M3 symmetric; M4 antisymmetric
  O[4] = -eS * m2_21 - eH * m3_21 + eQ * m4_21;
  O[1] = -eS * m2_21 - eH * m3_21 - eQ * m4_21;
  O[8] = -eS * m2_31 - eH * m3_31 + eQ * m4_31;
  O[2] = -eS * m2_31 - eH * m3_31 - eQ * m4_31;
  O[12] = -eS * m2_41 - eH * m3_41 + eQ * m4_41;
  O[3] = -eS * m2_41 - eH * m3_41 - eQ * m4_41;
  // (3,2),(2,3): M2,M3 antisymmetric; M4 symmetric
  O[9] = -eS * m2_32 - eH * m3_32 + eQ * m4_32;
  O[6] = eS * m2_32 + eH * m3_32 + eQ * m4_32;
  O[13] = -eS * m2_42 - eH * m3_42 + eQ * m4_42;
  O[7] = eS * m2_42 + eH * m3_42 + eQ * m4_42;
  O[14] = -eS * m2_43 - eH * m3_43 + eQ * m4_43;
  O[11] = eS * m2_43 + eH * m3_43 + eQ * m4_43;
}

}  // namespace fzd
