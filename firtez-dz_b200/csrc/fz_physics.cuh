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
#include "fz_pftable.h"

namespace fzd {

// ------------------------------------------------------------------ constants
struct Consts {
  double csaha1, csaha2, rbohr, deno_sa, deno_sam;
  double ab10[FZ_NELEM];   // 10**(ABUND-12)
  // element handled by lane l in slot j of the warp chemistry: lane_elem[32*j+l]
  // (-1 = idle).  Slot 0 holds every element whose partition function has an
  // exponential piece, so slots 1 and 2 never evaluate one.
  int lane_elem[96];
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

// Horner with fused multiply-adds (the FP64 chemistry kernels evaluate the
// pieces millions of times; the unfused form of horner_exact is kept for the
// per-line opacities, which follow the reference's rounding step by step).
__device__ __forceinline__ double horner6(const double* c, double x) {
  double r = c[5];
  r = fma(x, r, c[4]);
  r = fma(x, r, c[3]);
  r = fma(x, r, c[2]);
  r = fma(x, r, c[1]);
  r = fma(x, r, c[0]);
  return r;
}

// U of one (element, stage) without divergent branches: the active piece
// (the last whose condition holds) is selected by predication, then one
// Horner evaluation and one exponential (used only by exp forms).
template <bool EXPF>
__device__ __forceinline__ double pf_stage(const PFTable* __restrict__ tb, int e, int s, double T,
                                           const double var[3]) {
  const int nv = tb->nv[e][s];
  int act = 0;
#pragma unroll
  for (int i = 1; i < FZ_PF_MAXV; ++i) {
    const int cond = __ldg(&tb->p[e][s][i].cond);
    const double th = __ldg(&tb->p[e][s][i].th);
    const bool ok = (cond == 1 && T > th) || (cond == 2 && T < th) || (cond == 3 && T <= th) || (cond == 4 && T >= th);
    act = (i < nv && ok) ? i : act;
  }
  const PFPiece* p = &tb->p[e][s][act];
  double c[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) c[i] = __ldg(&p->c[i]);
  const int form = __ldg(&p->form), v = __ldg(&p->var);
  const double x = v == 0 ? var[0] : (v == 1 ? var[1] : var[2]);
  const double h = horner6(c, x);
  double u = h;
  if (EXPF) u = form == 1 ? __ldg(&p->base) + exp(h) : u;
  u = form == 2 ? fmax(__ldg(&p->clamp), h) : u;
  return nv > 0 ? u : 0.0;
}

// U_I, U_II, U_III of element zn (1-based), src/atom_database.f90:121-1035
// (generated piece table; branchy, used outside the warp chemistry).
__device__ __forceinline__ double pf_vpiece(const fz_pf_vpiece& p, const double var[3]) {
  const double h = horner_exact(p.c, p.nc, var[p.var]);
  if (p.form == 1) return p.base + exp(h);
  if (p.form == 2) return fmax(p.clamp, h);
  return h;
}

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

// 1/y to ~1 ulp: hardware approximation refined by two Newton steps.
__device__ __forceinline__ double rcp_d(double y) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(y));
  double e = fma(-y, r, 1.0);
  r = fma(r, e, r);
  e = fma(-y, r, 1.0);
  return fma(r, e, r);
}

// --------------------------------------------------------- warp chemistry
// One column's chemistry on a group of L lanes (L = 32: a warp; L = 16: a
// half-warp, two columns per warp), lanes over the elements: the element of
// lane l in slot j is lane_elem[L*j + l], NS = 96 / L slots per lane.  The
// exponential-form elements come first in lane_elem, so only the first
// 32 / L slots of a lane (the first 32 of the 96) evaluate an exponential.
template <int L>
struct WarpSahaT {
  static constexpr int NS = 96 / L;
  double T;
  double a1[NS], a2[NS];
  unsigned hyd;   // bit j: the lane's slot j holds hydrogen
};
using WarpSaha = WarpSahaT<32>;

__device__ __forceinline__ double clamp650(double e) {
  if (e > 0.0) e = fmin(e, 650.0);
  if (e < 0.0) e = fmax(e, -650.0);
  return e;
}

// The temperature terms the Saha factors of every element share: 1/T,
// T^(-3/2) x CSAHA1 and the partition functions' variables (T, T/1000,
// log(5040/T)).
struct SahaT {
  double it, lamelec, var[3];
};

__device__ __forceinline__ SahaT saha_t(double T, const Consts& K) {
  SahaT t;
  t.it = rcp_d(T);
  t.lamelec = K.csaha1 * (t.it * sqrt(t.it));   // T^(-3/2)
  t.var[0] = T;
  t.var[1] = 1.0e-3 * T;
  t.var[2] = log(5040.0 / T);
  return t;
}

// The Saha factors (a1, a2) of element el (-1: an idle slot, (0, 0)) at
// temperature T (SHORT_PRE_ION_CALC_TEMPRHO, src/chemical_equilibrium.f90:
// 1601-1652).  EXPF: the element's partition-function pieces may hold an
// exponential (every such element sits in the first 32 slots).
template <bool EXPF>
__device__ __forceinline__ double2 saha_elem(int el, double T, const SahaT& t, const Consts& K,
                                             const PFTable* __restrict__ tb) {
  const int e = el < 0 ? 0 : el;
  const double u0 = pf_stage<EXPF>(tb, e, 0, T, t.var);
  const double u1 = pf_stage<EXPF>(tb, e, 1, T, t.var);
  const double u2 = pf_stage<EXPF>(tb, e, 2, T, t.var);
  const double e1 = exp(clamp650(K.csaha2 * fz_tab_xi[e] * t.it));
  const double e2 = exp(clamp650(K.csaha2 * fz_tab_xii[e] * t.it));
  return make_double2(el >= 0 ? (u0 * (0.5 * rcp_d(u1))) * t.lamelec * e1 : 0.0,
                      el >= 0 ? (u1 * (0.5 * rcp_d(u2))) * t.lamelec * e2 : 0.0);
}

// Bit j of the lane's hydrogen mask: its slot j holds hydrogen.
template <int L>
__device__ __forceinline__ unsigned saha_hyd(const Consts& K, int lane) {
  unsigned h = 0u;
#pragma unroll
  for (int j = 0; j < WarpSahaT<L>::NS; ++j)
    if (K.lane_elem[L * j + lane] == 0) h |= 1u << j;
  return h;
}

// Per-lane Saha factors of the lane's elements at temperature T
// (SHORT_PRE_ION_CALC_TEMPRHO, src/chemical_equilibrium.f90:1601-1652): the
// arithmetic of saha_t + saha_elem written inline (so the chain's register
// allocation stays as it was), bit for bit the same values.
template <int L>
__device__ __forceinline__ void saha_prepare(WarpSahaT<L>& w, double T, const Consts& K,
                                             const PFTable* __restrict__ tb, int lane) {
  constexpr int NS = WarpSahaT<L>::NS;
  constexpr int NEXP = 32 / L;   // the lane's slots among the first 32 (the 23 exponential-form elements)
  w.T = T;
  w.hyd = 0u;
  const double it = rcp_d(T);
  const double lamelec = K.csaha1 * (it * sqrt(it));   // T^(-3/2)
  const double var[3] = {T, 1.0e-3 * T, log(5040.0 / T)};
#pragma unroll
  for (int j = 0; j < NS; ++j) {
    const int el = K.lane_elem[L * j + lane];
    const int e = el < 0 ? 0 : el;
    double u0, u1, u2;
    if (j < NEXP) {
      u0 = pf_stage<true>(tb, e, 0, T, var);
      u1 = pf_stage<true>(tb, e, 1, T, var);
      u2 = pf_stage<true>(tb, e, 2, T, var);
    } else {
      u0 = pf_stage<false>(tb, e, 0, T, var);
      u1 = pf_stage<false>(tb, e, 1, T, var);
      u2 = pf_stage<false>(tb, e, 2, T, var);
    }
    const double e1 = exp(clamp650(K.csaha2 * fz_tab_xi[e] * it));
    const double e2 = exp(clamp650(K.csaha2 * fz_tab_xii[e] * it));
    if (el == 0) w.hyd |= 1u << j;
    w.a1[j] = el >= 0 ? (u0 * (0.5 * rcp_d(u1))) * lamelec * e1 : 0.0;
    w.a2[j] = el >= 0 ? (u1 * (0.5 * rcp_d(u2))) * lamelec * e2 : 0.0;
  }
}


// The lane's Saha factors of one temperature sample from a precomputed row
// (96 slots of (a1, a2) in slot order, k_saha).
template <int L>
__device__ __forceinline__ void saha_load(WarpSahaT<L>& w, double T, unsigned hyd, const double2* __restrict__ row,
                                          int lane) {
  w.T = T;
  w.hyd = hyd;
#pragma unroll
  for (int j = 0; j < WarpSahaT<L>::NS; ++j) {
    const double2 a = __ldcs(row + L * j + lane);
    w.a1[j] = a.x;
    w.a2[j] = a.y;
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;   // xor butterfly: bit-identical in every lane
}

// Sum over the L lanes of a group (xor butterfly within the group; mask:
// the group's lanes).
template <int L>
__device__ __forceinline__ double group_sum(double v, unsigned mask) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}

// The lanes of this thread's group of L.
template <int L>
__device__ __forceinline__ unsigned group_mask() {
  return L == 32 ? 0xffffffffu : (((1u << L) - 1u) << (threadIdx.x & 31 & ~(L - 1)));
}

struct RhoOut {
  double nhyd, pelec, dens, molecw;
  int status;
};

// GET_RHO, src/chemical_equilibrium.f90:165-278.  All lanes of the group
// call it with the same arguments; nelec (the warm-start chain) is updated in
// every lane identically.  The electron sum of SHORT_ION_CALC_TEMPRHO
// (:1659-1701), NELEC_EST = N_H+ - N_H- + sum_{Z>1} (N_II + N_III), is
// evaluated per element as ab*(1+y)/(1+y+xy) (hydrogen: ab*(1-xy)/(1+y+xy))
// with x = ne*alpha_I, y = ne*alpha_II: algebraically the reference's three
// quotients, one division instead of five.  ab[j] = 10**(ABUND-12) of the
// lane's elements (0 past element 92).
template <int L>
__device__ __forceinline__ RhoOut get_rho_warp(const WarpSahaT<L>& w, const double ab[WarpSahaT<L>::NS], double PG,
                                               double& nelec, const Consts& K, int lane) {
  constexpr int NS = WarpSahaT<L>::NS;
  const unsigned mask = group_mask<L>();
  RhoOut r;
  const double T = w.T;
  double nhyd = 0.0;
  if (nelec != nelec) nelec = 0.0;
  if (nelec < 1.0) nelec = PG / (101.0 * KBOL * T);
  const double pelec = nelec * KBOL * T;
  if (pelec > PG) nelec = (PG * 0.5) / (KBOL * T);
  int iter = 1;
  double nnew = nelec, nold = nelec;
  const double kt = KBOL * T, idkt = rcp_d(K.deno_sa * KBOL * T);
  bool go = true;
  while (go) {
    nold = nnew;
    nhyd = (PG - nnew * kt) * idkt;
    const double ne = nnew;
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < NS; ++j) {
      const double x = ne * w.a1[j], y = ne * w.a2[j];
      const double xy = x * y;
      const double num = ((w.hyd >> j) & 1u) ? (1.0 - xy) : (1.0 + y);   // hydrogen: N_H+ - N_H-
      s = fma(ab[j] * num, rcp_d(1.0 + y + xy), s);
    }
    s = group_sum<L>(s, mask);
    const double est = nhyd * s;
    nnew = (fmax(est, 0.0) + nold) * 0.5;
    iter = iter + 1;
    // ERROR = |(NEW-OLD)/NEW| > 1e-4, ITER <= 100, NHYD >= 0
    go = fabs(nnew - nold) > 1.0e-4 * fabs(nnew) && iter <= 100 && nhyd >= 0.0;
  }
  r.status = 0;
  if (iter >= 100 || nhyd < 0.0) r.status = 1;
  nelec = nnew;
  nhyd = (PG - nelec * KBOL * T) * idkt;
  r.dens = nhyd * K.deno_sam + nelec * MELE;
  r.molecw = ((r.dens * KBOL * T) * (1.0 / MAMU)) * rcp_d(PG);
  if (nhyd != nhyd || nnew != nnew) r.status = 2;
  if (nelec < 0.0 || nhyd <= 0.0) r.status = 1;
  r.nhyd = nhyd;
  r.pelec = pelec;   // pressure of the initial guess, as the reference returns it
  return r;
}

// ----------------------------------------------------- continuum opacity
// OPAC_CONTINUUM, src/cont_opacity.f90:305-357, with every factor that
// depends only on the wavelength precomputed on the host (ContP):
//   H- free-free  (:48-120):  1e-29 k ne T sum_i c_i theta^(1+i/2)
//   H- bound-free (:124-181): T^-2.5 e^(a1/T) (1 - e^(-a2/T)) sigma ne k T
//   Thomson (:187-217), Rayleigh (:221-239), neutral H bf/ff (:243-301).
struct ContP {
  int nff, n0, pad0, pad1;
  double ffc[6];
  double sbf, bfa1, bfa2;        // sigma_bf (0 if lambda >= 1.6419 um), ALPHA/LAMBDAP, ALPHA/lambda_um
  double hpre, c3l, c4, ray;     // C2 lambda^3, C3/lambda, C4, Rayleigh
  double ct;                     // Thomson constant
};

__device__ __forceinline__ double opac_continuum(double T, double ne, double nh, const ContP& c) {
  const double th = 5040.0 / T;
  const double sq = sqrt(th);
  const double th2 = th * th;
  double part1 = c.ffc[0] * th + c.ffc[1] * th * sq + c.ffc[2] * th2 + c.ffc[3] * th2 * sq;
  if (c.nff == 6) part1 += c.ffc[4] * th2 * th + c.ffc[5] * th2 * th * sq;
  const double hmff = 1e-29 * part1 * KBOL * ne * T;
  double hmbf = 0.0;
  if (c.sbf != 0.0) {
    const double part = (1.0 / (T * T * sqrt(T))) * exp(c.bfa1 / T) * (1.0 - exp(-c.bfa2 / T));
    hmbf = part * c.sbf * ne * KBOL * T;
  }
  const double thom = c.ct * (ne / nh);
  double sum;
  if (c.n0 <= 8) {
    sum = 0.0;
    for (int i = c.n0; i <= 8; ++i) {
      const double di = (double)i;
      sum += exp(c.c4 / (T * di * di)) / (di * di * di);
    }
    sum += (0.117 + exp(c.c4 / (T * 81.0))) * (T / (2.0 * c.c4));
  } else {
    const double dn = (double)c.n0;
    sum = (0.117 + exp(c.c4 / (T * dn * dn))) * (T / (2.0 * c.c4));
  }
  const double hyd = c.hpre * sum * (1.0 - exp(-c.c3l / T)) * exp(-c.c4 / T);
  return nh * (hmff + hmbf + thom + c.ray + hyd);
}

// ------------------------------------------------------ line opacity, damping
// Per-line constants precomputed on the host.
struct LineP {
  double l0, wdif;
  double term1;      // TERM1 of OPAC_LINE, src/line_opacity.f90:95
  double m2k;        // matom m_u / (2 k): TERM2 = sqrt(m2k / T)
  double chik;       // EPLOW e / k:        TERM4 = exp(-chik / T)
  double hclk;       // h c / (lambda k):   TERM5 = 1 - exp(-hclk / T)
  double nab;        // 10**(ABUND-12)
  double xi_k, xii_k;    // CSAHA2 * XI, XII of the element
  double vdk;        // 2 k / (m_u matom): v_D = sqrt(vdk T)
  double grad;       // radiative damping 0.2223 / lambda^2
  double gc, ge;     // collisional: gamma_col = gc nH T^ge
  double dfac;       // lambda / (4 pi)
  int zn, ion;
};

// OPAC_LINE (LTE) with ION_CALC_TEMPX, src/line_opacity.f90:34-108,
// src/chemical_equilibrium.f90:1511-1597.
__device__ __forceinline__ double opac_line(const LineP& L, double T, double ne, double nh, const Consts& K) {
  const double var[3] = {T, 1.0e-3 * T, log(5040.0 / T)};
  double U[3];
  partition_u(L.zn, T, var, U);
  const double lamelec = K.csaha1 / (T * sqrt(T));
  const double al1 = (U[0] / (2.0 * U[1])) * lamelec * exp(clamp650(L.xi_k / T));
  const double al2 = (U[1] / (2.0 * U[2])) * lamelec * exp(clamp650(L.xii_k / T));
  const double deno = ne * ne * al1 * al2 + ne * al2 + 1.0;
  const double nume = L.ion == 1 ? ne * ne * al1 * al2 : (L.ion == 2 ? ne * al2 : 1.0);
  const double npi = nh * L.nab * nume / deno;
  const double t2 = sqrt(L.m2k / T);
  const double t4 = exp(-L.chik / T);
  const double t5 = 1.0 - exp(-L.hclk / T);
  return L.term1 * t2 * (npi / U[L.ion - 1]) * t4 * t5;
}

// GET_DAMPING, src/damping.f90:842-1012: a = (gamma_rad + gamma_col) lambda / (4 pi v_D)
__device__ __forceinline__ double get_damping(const LineP& L, double nh, double T) {
  const double gcol = L.gc * nh * pow(T, L.ge);
  return (L.grad + gcol) * L.dfac / sqrt(L.vdk * T);
}

// ------------------------------------------------------------ FP32 Voigt
// Hui, Armstrong & Wray (1978) 7-pole rational approximation of the complex
// probability function, as src/voigt.f:17-98: H = Re w, F = sign(v) Im w
// with w = P(z)/Q(z) at z = a - i|v|.  P (degree 6) and Q (monic, degree 7)
// have real coefficients, so each is reduced modulo the real quadratic
// (z^2 - 2 Re z z + |z|^2) that z solves (Knuth, TAOCP vol. 2, 4.6.4):
// 2 FMA per degree instead of a complex multiply-add.  The quotient is
// P conj(Q') sc / |Q'|^2 with Q' = Q sc, sc = 1 / max(|Re Q|, |Im Q|), so
// |Q'|^2 lies in [1, 2] whatever the size of Q (an error in sc cancels);
// its reciprocals are the approximate ones (a few ulp in all, far inside
// the approximation's own error) and no compare or select is needed.
__device__ __forceinline__ void voigt_f32(float a, float u, float& H, float& F) {
  const float A0 = 122.607931777104326f, A1 = 214.382388694706425f, A2 = 181.928533092181549f,
              A3 = 93.155580458138441f, A4 = 30.180142196210589f, A5 = 5.912626209773153f,
              A6 = .564189583562615f, B0 = 122.60793177387535f, B1 = 352.730625110963558f,
              B2 = 457.334478783897737f, B3 = 348.703917719495792f, B4 = 170.354001821091472f,
              B5 = 53.992906912940207f, B6 = 10.479857114260399f;
  const float v = fabsf(u);
  const float x = a, y = -v;
  const float r = 2.0f * x, s = fmaf(x, x, v * v);
  float p1 = A6, p0 = A5, t;
#define FZ_KSTEP(C, hi, lo) \
  t = hi;                   \
  hi = fmaf(r, t, lo);      \
  lo = fmaf(-s, t, (C));
  FZ_KSTEP(A4, p1, p0) FZ_KSTEP(A3, p1, p0) FZ_KSTEP(A2, p1, p0) FZ_KSTEP(A1, p1, p0) FZ_KSTEP(A0, p1, p0)
  float q1 = 1.0f, q0 = B6;
  FZ_KSTEP(B5, q1, q0) FZ_KSTEP(B4, q1, q0) FZ_KSTEP(B3, q1, q0) FZ_KSTEP(B2, q1, q0) FZ_KSTEP(B1, q1, q0)
  FZ_KSTEP(B0, q1, q0)
#undef FZ_KSTEP
  // P = p1 z + p0, Q = q1 z + q0
  const float nr = fmaf(p1, x, p0), ni = p1 * y;
  const float dr = fmaf(q1, x, q0), di = q1 * y;
  const float sc = __fdividef(1.0f, fmaxf(fabsf(dr), fabsf(di)));
  const float dr1 = dr * sc, di1 = di * sc;
  const float k = sc * __fdividef(1.0f, fmaf(dr1, dr1, di1 * di1));
  const float wr = fmaf(nr, dr1, ni * di1) * k;
  const float wi = fmaf(ni, dr1, -(nr * di1)) * k;
  H = wr;
  F = (u < 0.0f) ? -wi : wi;
}

// Evolution operator O of one layer from its optical-depth increments
// t = eta*dz (src/rtesolver.f90:269-473), and om0 = 1 - O(1,1).  The reference's clamp of cosh and
// sinh at 2^53 (-> 1e15, :464-465) is reproduced; below it the operator is
// evaluated with cancellation-free forms (cosh x -+ cos y via sinh^2(x/2),
// sin^2(y/2); lambda_1,2 from the larger root).
// The layer's scalars of the operator: |eta|^2, |rho|^2, eta.rho, their
// difference d, R = theta / 2, the roots x = lambda_1 dz and y = lambda_2
// dz, sign(eta.rho), 1/theta, e^-tI and the hyperbolic / trigonometric
// factors (P = cosh-like, Qm = sinh^2(x/2) + sin^2(y/2), sh = sinh x,
// s2v = sin y, c2v = cos y, ch = cosh x, amb = P - 1).
struct EvolCore {
  float eta2, rho2, er, d, R, x, y, sg, it, E, P, Qm, sh, s2v, c2v, ch, amb;
  bool clamp;
};

__device__ __forceinline__ void evol_core(float tI, float tQ, float tU, float tV, float rQ, float rU, float rV,
                                          EvolCore& c) {
  c.eta2 = tQ * tQ + tU * tU + tV * tV;
  c.rho2 = rQ * rQ + rU * rU + rV * rV;
  c.er = tQ * rQ + tU * rU + tV * rV;
  c.d = c.eta2 - c.rho2;
  c.R = sqrtf(0.25f * c.d * c.d + c.er * c.er);
  if (c.d >= 0.0f) {
    c.x = sqrtf(c.R + 0.5f * c.d);
    c.y = c.x > 0.0f ? fabsf(c.er) / c.x : 0.0f;
  } else {
    c.y = sqrtf(c.R - 0.5f * c.d);
    c.x = c.y > 0.0f ? fabsf(c.er) / c.y : 0.0f;
  }
  c.sg = c.er > 0.0f ? 1.0f : (c.er < 0.0f ? -1.0f : 0.0f);
  const float theta = 2.0f * c.R;
  c.it = theta > 0.0f ? 1.0f / theta : 0.0f;
  c.E = expf(-tI);
  const float XCLAMP = 37.42994775f;   // cosh, sinh >= 2^53 in float64
  c.amb = 0.0f;
  c.s2v = sinf(c.y);
  c.clamp = c.x >= XCLAMP;
  if (c.clamp) {
    const float c2 = cosf(c.y);
    c.P = 0.5f * (1e15f + c2);
    c.Qm = 0.5f * (1e15f - c2);
    c.sh = 1e15f;
    c.ch = 1e15f;
    c.c2v = c2;
  } else {
    const float shx = sinhf(0.5f * c.x), siy = sinf(0.5f * c.y);
    const float a = shx * shx, b = siy * siy;
    c.amb = a - b;
    c.P = 1.0f + c.amb;
    c.Qm = a + b;
    c.sh = sinhf(c.x);
    c.ch = 1.0f + 2.0f * a;
    c.c2v = 1.0f - 2.0f * b;
  }
}

// O and om0 = 1 - O(1,1) from the layer's scalars.
__device__ __forceinline__ void evol_matrix(const EvolCore& c, float tI, float tQ, float tU, float tV, float rQ,
                                            float rU, float rV, float O[16], float& om0) {
  const float x = c.x, y = c.y, sg = c.sg, it = c.it;
  // M2, M3, M4 (Fortran (row,col) -> O[4*(row-1)+(col-1)])
  const float m2_21 = (y * tQ - sg * x * rQ) * it, m2_31 = (y * tU - sg * x * rU) * it,
              m2_41 = (y * tV - sg * x * rV) * it;
  const float m2_32 = (sg * x * tV + y * rV) * it, m2_42 = (-sg * x * tU - y * rU) * it,
              m2_43 = (sg * x * tQ + y * rQ) * it;
  const float m3_21 = (x * tQ + sg * y * rQ) * it, m3_31 = (x * tU + sg * y * rU) * it,
              m3_41 = (x * tV + sg * y * rV) * it;
  const float m3_32 = (-sg * y * tV + x * rV) * it, m3_42 = (sg * y * tU - x * rU) * it,
              m3_43 = (-sg * y * tQ + x * rQ) * it;
  const float m4_11 = (c.eta2 + c.rho2) * it;   // 2*((eta2+rho2)/2)/theta
  const float m4_21 = 2.0f * (tV * rU - tU * rV) * it, m4_31 = 2.0f * (tQ * rV - tV * rQ) * it,
              m4_41 = 2.0f * (tU * rQ - tQ * rU) * it;
  const float m4_22 = 2.0f * (tQ * tQ + rQ * rQ) * it - m4_11, m4_33 = 2.0f * (tU * tU + rU * rU) * it - m4_11,
              m4_44 = 2.0f * (tV * tV + rV * rV) * it - m4_11;
  const float m4_32 = 2.0f * (tQ * tU + rQ * rU) * it, m4_42 = 2.0f * (tV * tQ + rV * rQ) * it,
              m4_43 = 2.0f * (tU * tV + rU * rV) * it;
  const float E = c.E;
  const float eP = E * c.P, eQ = E * c.Qm, eS = E * c.s2v, eH = E * c.sh;
  O[0] = eP + eQ * m4_11;
  // 1 - O(1,1) without cancellation in optically thin layers:
  // (1 - e^-tI) - e^-tI (P - 1 + Qm M4(1,1))
  om0 = c.clamp ? 1.0f - O[0] : -expm1f(-tI) - E * (c.amb + c.Qm * m4_11);
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

__device__ __forceinline__ void evol_f32(float tI, float tQ, float tU, float tV, float rQ, float rU, float rV,
                                         float O[16], float& om0) {
  EvolCore c;
  evol_core(tI, tQ, tU, tV, rQ, rU, rV, c);
  evol_matrix(c, tI, tQ, tU, tV, rQ, rU, rV, O, om0);
}

}  // namespace fzd
