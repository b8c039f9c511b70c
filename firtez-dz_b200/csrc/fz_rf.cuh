// Device physics of the response functions (sm_100a).
//
//  * FP64, one warp per (column, height): the chemistry derivatives of
//    GET_DNHYDDTEMP (src/chemical_equilibrium.f90:2008-2052) at constant Pg
//    and T, and the T|Pg and Pg|T derivatives of the continuum opacity
//    (src/cont_opacity.f90:48-357), line opacity (src/line_opacity.f90:109-207)
//    and damping (src/damping.f90:878-1008).
//  * FP32, one thread per wavelength: directional derivatives of the
//    evolution operator (src/rtesolver.f90:476-1002) written on per-layer
//    optical depths, in vector form.
#pragma once
#include "fz_physics.cuh"

namespace fzd {

// U and dlnU/dT of every stage of element e (0-based) from the generated
// piece tables (src/atom_database.f90:121-1035).
__device__ __forceinline__ void partition_udu(int e, double T, double U[3], double dU[3]) {
  const double var[3] = {T, 1.0e-3 * T, log(5040.0 / T)};
#pragma unroll 1
  for (int s = 0; s < 3; ++s) {
    const int nv = fz_tab_pf_nv[e][s];
    int act = -1;
    for (int i = 0; i < nv; ++i)
      if (pf_cond(fz_tab_pf_v[e][s][i].cond, fz_tab_pf_v[e][s][i].th, T, 0.0)) act = i;
    U[s] = act >= 0 ? pf_vpiece(fz_tab_pf_v[e][s][act], var) : 0.0;
    double d = 0.0;
    const int nd = fz_tab_pf_nd[e][s];
    for (int i = 0; i < nd; ++i) {
      const fz_pf_dpiece& p = fz_tab_pf_d[e][s][i];
      const double uref = p.ref >= 0 ? pf_vpiece(fz_tab_pf_v[e][s][p.ref], var) : U[s];
      if (!pf_cond(p.cond, p.th, T, uref)) continue;
      double h = horner_exact(p.c, p.nc, var[p.var]) * p.mult;
      for (int k = 0; k < p.dx; ++k) h *= (-1.0 / T);
      if (p.ub) h *= (uref - p.base);
      for (int k = 0; k < p.up; ++k) h /= uref;
      d = h;
    }
    dU[s] = d;
  }
}

// Saha factors alpha_I, alpha_II of element e and their T-derivatives
// (ION_CALC_TEMPPGAS, src/chemical_equilibrium.f90:1812-1842).
struct Alpha {
  double a1, a2, da1, da2;
  double U[3], dU[3];
};

__device__ __forceinline__ Alpha alpha_of(int e, double T, const Consts& K) {
  Alpha a;
  partition_udu(e, T, a.U, a.dU);
  const double lamelec = K.csaha1 * pow(T, -3.0 / 2.0);
  const double e1 = exp(clamp650(K.csaha2 * fz_tab_xi[e] / T));
  const double e2 = exp(clamp650(K.csaha2 * fz_tab_xii[e] / T));
  a.a1 = (a.U[0] / (2.0 * a.U[1])) * lamelec * e1;
  a.a2 = (a.U[1] / (2.0 * a.U[2])) * lamelec * e2;
  const double dlam = -3.0 / (2.0 * T);
  const double it2 = 1.0 / (T * T);
  a.da1 = a.a1 * (a.dU[0] - a.dU[1] + dlam - K.csaha2 * fz_tab_xi[e] * it2);
  a.da2 = a.a2 * (a.dU[1] - a.dU[2] + dlam - K.csaha2 * fz_tab_xii[e] * it2);
  return a;
}

struct ChemDer {
  double dne_p, dnh_p;   // DNELECDPG_TEMP, DNHYDDPG_TEMP
  double dne_t, dnh_t;   // DNELECDTEMP_PG, DNHYDDTEMP_PG
};

__device__ __forceinline__ double sel3(const double v[3], int i) { return i == 0 ? v[0] : (i == 1 ? v[1] : v[2]); }

// U and dlnU/dT of one (element, stage) from the padded device tables, with
// lanes on different elements: every value piece is evaluated once (the
// derivative pieces' conditions and factors refer to them), the active value
// and derivative pieces are selected by predication, and only the active
// derivative piece is evaluated.  Same pieces, Horner order and rounded -1/T
// as partition_udu; the Horner steps are fused (last-bit differences).
__device__ __forceinline__ void pf_stage_udu(const PFTable* __restrict__ tb, const PFDTable* __restrict__ td, int e,
                                             int s, double T, double it, const double var[3], double& U,
                                             double& dU) {
  const int nv = __ldg(&tb->nv[e][s]);
  double vals[FZ_PF_MAXV];
  int act = 0;
#pragma unroll
  for (int i = 0; i < FZ_PF_MAXV; ++i) {
    const PFPiece* p = &tb->p[e][s][i];
    double u = 0.0;
    if (i < nv) {
      double c[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) c[k] = __ldg(&p->c[k]);
      const int form = __ldg(&p->form), v = __ldg(&p->var);
      const double h = horner6(c, v == 0 ? var[0] : (v == 1 ? var[1] : var[2]));
      u = h;
      if (form == 1) u = __ldg(&p->base) + exp(h);
      if (form == 2) u = fmax(__ldg(&p->clamp), h);
      if (i > 0) {
        const int cond = __ldg(&p->cond);
        const double th = __ldg(&p->th);
        const bool ok = (cond == 1 && T > th) || (cond == 2 && T < th) || (cond == 3 && T <= th) ||
                        (cond == 4 && T >= th);
        act = ok ? i : act;
      }
    }
    vals[i] = u;
  }
  U = nv > 0 ? sel3(vals, act) : 0.0;
  const int nd = __ldg(&td->nd[e][s]);
  int dact = -1;
  double uref = U;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const PFDPiece* p = &td->d[e][s][i];
    const int cond = __ldg(&p->cond), ref = __ldg(&p->ref);
    const double th = __ldg(&p->th);
    const double ur = ref < 0 ? U : sel3(vals, ref);
    const bool ok = i < nd && (cond == 0 || (cond == 1 && T > th) || (cond == 2 && T < th) ||
                               (cond == 3 && T <= th) || (cond == 4 && T >= th) || (cond == 5 && ur != th));
    dact = ok ? i : dact;
    uref = ok ? ur : uref;
  }
  double d = 0.0;
  if (dact >= 0) {
    const PFDPiece* p = &td->d[e][s][dact];
    double c[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) c[k] = __ldg(&p->c[k]);
    const int v = __ldg(&p->var);
    double h = horner6(c, v == 0 ? var[0] : (v == 1 ? var[1] : var[2])) * __ldg(&p->mult);
    if (__ldg(&p->dx)) h *= -it;
    if (__ldg(&p->ub)) h *= (uref - __ldg(&p->base));
    if (__ldg(&p->up)) h /= uref;
    d = h;
  }
  dU = d;
}

// GET_NE_TEMP_SNE_ALT (:892-957) and GET_DNE_PG (:2062-2155) by one warp,
// lanes over the elements.  In GET_DNE_PG every element's term of the sum is
// affine in the trial derivative DNE (ION_CALC_TEMPPGAS, :1791-1872), so the
// sum is A + B*DNE with A, B reduced once; the reference's damped fixed
// point (tolerance 1e-6, <= 101 passes) then runs on these two scalars with
// its own update and stopping rules.  The per-element algebra of
// ION_CALC_NETEMP_NEW (:1376-1442) and ION_CALC_TEMPPGAS is written on the
// reciprocals 1/(NE a_I), 1/(NE a_II), 1/x_1..3 and 1/DENOI (eight divisions
// instead of some forty); the T-only factors are taken once per warp.
__device__ __forceinline__ ChemDer chem_der_warp(double T, double P, double NE, const Consts& K,
                                                 const PFTable* __restrict__ tb, const PFDTable* __restrict__ td,
                                                 int lane) {
  const double it = 1.0 / T;
  const double ideno = 1.0 / K.deno_sa;
  const double nh = (P - NE * KBOL * T) * (it / KBOL) * ideno;
  const double var[3] = {T, 1.0e-3 * T, log(5040.0 / T)};
  const double lamelec = K.csaha1 * (it * sqrt(it));   // T^(-3/2)
  const double dlam = -1.5 * it;
  const double it2 = it * it;
  const double ine = 1.0 / NE;
  const double ne2 = NE * NE, ine2 = ine * ine;
  const double pk = P * it2 / KBOL;
  double sn = 0.0, sd = 0.0, sa = 0.0, sb = 0.0;
#pragma unroll 1
  for (int j = 0; j < 3; ++j) {
    const int e = K.lane_elem[32 * j + lane];
    if (e < 0) continue;
    double U[3], dU[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) pf_stage_udu(tb, td, e, s, T, it, var, U[s], dU[s]);
    const double xi = __ldg(&fz_tab_xi[e]), xii = __ldg(&fz_tab_xii[e]);
    const double e1 = exp(clamp650(K.csaha2 * xi * it));
    const double e2 = exp(clamp650(K.csaha2 * xii * it));
    const double a1 = (U[0] / (2.0 * U[1])) * lamelec * e1;
    const double a2 = (U[1] / (2.0 * U[2])) * lamelec * e2;
    const double da1 = a1 * (dU[0] - dU[1] + dlam - K.csaha2 * xi * it2);
    const double da2 = a2 * (dU[1] - dU[2] + dlam - K.csaha2 * xii * it2);
    const double ab = K.ab10[e];
    const double n = nh * ab;
    const double p1 = NE * a1, p2 = NE * a2;
    const double ip1 = 1.0 / p1, ip2 = 1.0 / p2;
    const double ia1 = NE * ip1, ia2 = NE * ip2;
    const double f1 = 1.0 / (1.0 + ip1 * (1.0 + ip2));   // ni / n
    const double f2 = 1.0 / (p1 + 1.0 + ip2);            // nii / n
    const double f3 = 1.0 / (1.0 + p2 * (p1 + 1.0));     // niii / n
    const double ni = n * f1, nii = n * f2, niii = n * f3;
    const double idn = 1.0 / ((p1 + 1.0) * p2 + 1.0);
    const double g = 2.0 * a1 * a2 * NE + a2;
    const double r = ab * ideno;
    const double rk = r * it / KBOL;
    // ION_CALC_NETEMP_NEW
    const double dn_i = f1 * rk, dn_ii = f2 * rk, dn_iii = f3 * rk;
    const double dd_i = -(f1 * r) + (n * (2.0 * a1 * a2 * NE) - ni * g) * idn;
    const double dd_ii = -(f2 * r) + (n * a2 - nii * g) * idn;
    const double dd_iii = -(f3 * r) - niii * g * idn;
    // ION_CALC_TEMPPGAS at DNE = 0 (A) and its DNE-coefficient (B)
    const double dn0 = -(r * pk);
    const double i1 = f1 * f1, i2 = f2 * f2, i3 = f3 * f3;
    const double q1 = n * i1 * (ine2 * ia1);
    const double dni0 = dn0 * f1 - q1 * ((-ia1) * (NE * da1) * (1.0 + ip2) - (ip2 * ia2) * (NE * da2));
    const double dni1 = -r * f1 - q1 * (-(1.0 + ip2) - ip2);
    const double dnii0 = dn0 * f2 - n * i2 * (NE * da1 - (NE * da2) * (ine2 * ia2 * ia2));
    const double dnii1 = -r * f2 - n * i2 * (a1 - ine2 * ia2);
    const double dniii0 = dn0 * f3 - n * i3 * (ne2 * da2 * a1 + ne2 * a2 * da1 + NE * da2);
    const double dniii1 = -r * f3 - n * i3 * (2.0 * NE * a1 * a2 + a2);
    if (e == 0) {   // hydrogen: N_H+ - N_H- (:1841-1846)
      sn += -dn_i + dn_iii;
      sd += -dd_i + dd_iii;
      sa += -dni0 + dniii0;
      sb += -dni1 + dniii1;
    } else {
      sn += dn_ii + dn_iii;
      sd += dd_ii + dd_iii;
      sa += dnii0 + dniii0;
      sb += dnii1 + dniii1;
    }
  }
  sn = warp_sum(sn);
  sd = warp_sum(sd);
  sa = warp_sum(sa);
  sb = warp_sum(sb);
  ChemDer c;
  c.dne_p = sn / (1.0 - sd);
  c.dnh_p = ideno * (it / KBOL - c.dne_p);
  double dold = 0.0, dnew = 0.0, derr = 1.0e20;
  int iter = 0;
  while (derr > 1e-6 && iter <= 100) {
    dold = dnew;
    dnew = ((sa + sb * dnew) + dold) / 2.0;
    if (fabs(dnew) > 1.0e40) dnew = 0.0;
    derr = fabs((dnew - dold) / dnew);
    iter = iter + 1;
  }
  c.dne_t = sa + sb * dnew;
  c.dnh_t = (-ideno) * (pk + c.dne_t);
  return c;
}

// d kc / dT at constant Pg and d kc / dPg at constant T of OPAC_CONTINUUM
// (src/cont_opacity.f90:48-357) on the host-precomputed factors of ContP.
// The hydrogen n0 > 8 branch keeps the reference's n = 9 in DSUM (:286-287).
__device__ __forceinline__ void cont_der(double T, double ne, double nh, const ContP& c, const ChemDer& cd,
                                         double& dkc_t, double& dkc_p) {
  const double th = 5040.0 / T;
  const double sq = sqrt(th);
  const double th2 = th * th;
  double part1 = c.ffc[0] * th + c.ffc[1] * th * sq + c.ffc[2] * th2 + c.ffc[3] * th2 * sq;
  double dp = c.ffc[0] + 1.5 * c.ffc[1] * sq + 2.0 * c.ffc[2] * th + 2.5 * c.ffc[3] * th * sq;
  if (c.nff == 6) {
    part1 += c.ffc[4] * th2 * th + c.ffc[5] * th2 * th * sq;
    dp += 3.0 * c.ffc[4] * th2 + 3.5 * c.ffc[5] * th2 * sq;
  }
  const double part2 = dp * (-th / T);
  const double ff = 1e-29 * part1 * KBOL * ne * T;
  const double dff_t = ff * (cd.dne_t / ne + 1.0 / T + part2 / part1);
  const double dff_p = ff / ne * cd.dne_p;
  double bf = 0.0, dbf_t = 0.0, dbf_p = 0.0;
  if (c.sbf != 0.0) {
    const double ea = exp(-c.bfa2 / T);
    const double part = (1.0 / (T * T * sqrt(T))) * exp(c.bfa1 / T) * (1.0 - ea);
    bf = part * c.sbf * ne * KBOL * T;
    const double dlp = (1.0 / T) * (-2.5 + (c.bfa2 - c.bfa1) / T - (c.bfa2 / T) * (1.0 / (1.0 - ea)));
    dbf_t = bf * (dlp + 1.0 / T + cd.dne_t / ne);
    dbf_p = bf / ne * cd.dne_p;
  }
  const double thom = c.ct * (ne / nh);
  const double dth_t = thom * (cd.dne_t / ne - cd.dnh_t / nh);
  const double dth_p = thom / ne * cd.dne_p - thom / nh * cd.dnh_p;
  const double it2 = 1.0 / (T * T);
  double sum, dsum;
  const double e81 = exp(c.c4 / (T * 81.0));
  if (c.n0 <= 8) {
    sum = 0.0;
    dsum = 0.0;
    for (int i = c.n0; i <= 8; ++i) {
      const double di = (double)i, d2 = di * di;
      const double ex = exp(c.c4 / (T * d2));
      sum += ex / (d2 * di);
      dsum -= c.c4 * ex / (d2 * d2 * di) * it2;
    }
    sum += (0.117 + e81) * (T / (2.0 * c.c4));
  } else {
    const double dn = (double)c.n0;
    sum = (0.117 + exp(c.c4 / (T * dn * dn))) * (T / (2.0 * c.c4));
    dsum = 0.0;
  }
  dsum += (1.0 / (2.0 * c.c4)) * (0.117 + e81) - (1.0 / (2.0 * 81.0 * T)) * e81;
  const double ec4 = exp(-c.c4 / T), ec3 = exp(-c.c3l / T);
  const double hyd = c.hpre * sum * (1.0 - ec3) * ec4;
  const double dhyd = hyd * (dsum / sum + c.c4 * it2) - (c.hpre * c.c3l * it2) * ec4 * ec3;
  const double factor = ff + bf + thom + c.ray + hyd;
  dkc_t = factor * cd.dnh_t + nh * (dff_t + dbf_t + dth_t + dhyd);
  dkc_p = factor * cd.dnh_p + nh * (dff_p + dbf_p + dth_p);
}

// KLIN and its derivatives (OPAC_LINE, src/line_opacity.f90:34-207 with
// ION_CALC_TEMPX :1511-1597 and ION_CALC_PGTEMP :1446-1507), written as
// klin times logarithmic derivatives of TERM2..TERM5.
__device__ __forceinline__ void line_der(const LineP& L, double T, double ne, double nh, const ChemDer& cd,
                                         const Consts& K, double& dkl_t, double& dkl_p) {
  const double klin = opac_line(L, T, ne, nh, K);
  const Alpha al = alpha_of(L.zn - 1, T, K);
  const double a1 = al.a1, a2 = al.a2, da1 = al.da1, da2 = al.da2;
  const double ne2 = ne * ne;
  const double deno = ne2 * a1 * a2 + ne * a2 + 1.0;
  const double ddeno_t = 2.0 * ne * cd.dne_t * a1 * a2 + ne2 * da1 * a2 + ne2 * a1 * da2 + cd.dne_t * a2 + ne * da2;
  const double ddeno_n = 2.0 * a1 * a2 * ne + a2;   // d deno / d ne
  double nume, dnume_t, dnume_n;
  if (L.ion == 1) {
    nume = ne2 * a1 * a2;
    dnume_t = 2.0 * ne * cd.dne_t * a1 * a2 + ne2 * da1 * a2 + ne2 * a1 * da2;
    dnume_n = 2.0 * a1 * a2 * ne;
  } else if (L.ion == 2) {
    nume = ne * a2;
    dnume_t = cd.dne_t * a2 + ne * da2;
    dnume_n = a2;
  } else {
    nume = 1.0;
    dnume_t = 0.0;
    dnume_n = 0.0;
  }
  // d ln N_PI / dT|Pg and the stage's d ln U / dT
  const double dln_npi_t = cd.dnh_t / nh + dnume_t / nume - ddeno_t / deno;
  const double dlnu = al.dU[L.ion - 1];
  const double t5 = 1.0 - exp(-L.hclk / T);
  const double dln_t = -0.5 / T + (dln_npi_t - dlnu) + L.chik / (T * T) - L.hclk / (T * T) * (1.0 - t5) / t5;
  dkl_t = klin * dln_t;
  // d ln N_PI / dPg|T = dnH/nH + d ln(FIR)/dne * dne/dPg
  dkl_p = klin * (cd.dnh_p / nh + (dnume_n / nume - ddeno_n / deno) * cd.dne_p);
}

// Damping derivatives (src/damping.f90:878-1008); gamma_col = gc nH T^ge in
// both the ABO and the Unsold branch.
__device__ __forceinline__ void damp_der(const LineP& L, double nh, double T, const ChemDer& cd, double& ddam_t,
                                         double& ddam_p) {
  const double tg = pow(T, L.ge);
  const double gcol = L.gc * nh * tg;
  const double pre = L.dfac / sqrt(L.vdk * T);   // lambda / (4 pi v_D)
  const double damp = (L.grad + gcol) * pre;
  const double dg_t = gcol * L.ge / T + L.gc * tg * cd.dnh_t;
  ddam_t = damp / (L.grad + gcol) * dg_t - damp * (0.5 / T);
  ddam_p = pre * gcol / nh * cd.dnh_p;
}

// ------------------------------------------------ FP32 evolution operator
// State of one layer's operator (per-layer optical depths t = eta*dz) kept
// for its directional derivatives.
struct EvolSt {
  float tQ, tU, tV, rQ, rU, rV;
  float d, er, R, x, y, sg, it;   // eta2-rho2, eta.rho, theta/2, lambda1, lambda2, sign, 1/theta
  float iv;                        // 1 / the larger root (x if d >= 0, else y; 0 when it is 0)
  float E, P, Qm, s2v, c2v, sh, ch;
};

// O and 1 - O(1,1) (as evol_f32) plus the state, from one evaluation of the
// layer's scalars.
__device__ __forceinline__ void evol_state(float tI, float tQ, float tU, float tV, float rQ, float rU, float rV,
                                           float O[16], float& om0, EvolSt& s) {
  EvolCore c;
  evol_core(tI, tQ, tU, tV, rQ, rU, rV, c);
  evol_matrix(c, tI, tQ, tU, tV, rQ, rU, rV, O, om0);
  s.tQ = tQ; s.tU = tU; s.tV = tV; s.rQ = rQ; s.rU = rU; s.rV = rV;
  s.d = c.d; s.er = c.er; s.R = c.R; s.x = c.x; s.y = c.y; s.sg = c.sg;
  s.it = c.it;   // 1/theta = 0.5/R
  const float root = c.d >= 0.0f ? c.x : c.y;
  s.iv = root > 0.0f ? 1.0f / root : 0.0f;
  s.E = c.E; s.P = c.P; s.Qm = c.Qm; s.s2v = c.s2v; s.c2v = c.c2v; s.sh = c.sh; s.ch = c.ch;
}

// X w = [eta.w~, eta w0 + rho x w~], Y w = [-rho.w~, -rho w0 + eta x w~]:
// the raw M2 = lambda2 X + sigma lambda1 Y and M3 = lambda1 X - sigma lambda2 Y
// of src/rtesolver.f90:367-405 applied to w.
__device__ __forceinline__ void xy_apply(float eQ, float eU, float eV, float rQ, float rU, float rV, const float w[4],
                                         float X[4], float Y[4]) {
  X[0] = eQ * w[1] + eU * w[2] + eV * w[3];
  X[1] = eQ * w[0] + (rU * w[3] - rV * w[2]);
  X[2] = eU * w[0] + (rV * w[1] - rQ * w[3]);
  X[3] = eV * w[0] + (rQ * w[2] - rU * w[1]);
  Y[0] = -(rQ * w[1] + rU * w[2] + rV * w[3]);
  Y[1] = -rQ * w[0] + (eU * w[3] - eV * w[2]);
  Y[2] = -rU * w[0] + (eV * w[1] - eQ * w[3]);
  Y[3] = -rV * w[0] + (eQ * w[2] - eU * w[1]);
}

// raw M4 (src/rtesolver.f90:407-436, before the factor 2/theta) applied to w
__device__ __forceinline__ void m4raw_apply(float eQ, float eU, float eV, float rQ, float rU, float rV, const float w[4],
                                            float M[4]) {
  const float h = 0.5f * (eQ * eQ + eU * eU + eV * eV + rQ * rQ + rU * rU + rV * rV);
  const float cQ = eU * rV - eV * rU, cU = eV * rQ - eQ * rV, cV = eQ * rU - eU * rQ;   // eta x rho
  const float ew = eQ * w[1] + eU * w[2] + eV * w[3], rw = rQ * w[1] + rU * w[2] + rV * w[3];
  M[0] = h * w[0] + (cQ * w[1] + cU * w[2] + cV * w[3]);
  M[1] = -cQ * w[0] + eQ * ew + rQ * rw - h * w[1];
  M[2] = -cU * w[0] + eU * ew + rU * rw - h * w[2];
  M[3] = -cV * w[0] + eV * ew + rV * rw - h * w[3];
}

// Products of the operator's matrices with one vector w, shared by every
// direction that uses w.
struct EvolW {
  float w[4], Xw[4], Yw[4], M2w[4], M3w[4], M4w[4], Ow[4];
};

__device__ __forceinline__ void evol_w(const EvolSt& s, const float O[16], const float w[4], EvolW& v) {
#pragma unroll
  for (int i = 0; i < 4; ++i) v.w[i] = w[i];
  xy_apply(s.tQ, s.tU, s.tV, s.rQ, s.rU, s.rV, w, v.Xw, v.Yw);
  float m4[4];
  m4raw_apply(s.tQ, s.tU, s.tV, s.rQ, s.rU, s.rV, w, m4);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    v.M2w[i] = (s.y * v.Xw[i] + s.sg * s.x * v.Yw[i]) * s.it;
    v.M3w[i] = (s.x * v.Xw[i] - s.sg * s.y * v.Yw[i]) * s.it;
    v.M4w[i] = 2.0f * m4[i] * s.it;
    v.Ow[i] = O[4 * i + 0] * w[0] + O[4 * i + 1] * w[1] + O[4 * i + 2] * w[2] + O[4 * i + 3] * w[3];
  }
}

// (dO/dt . dt) w for a direction dt = (dtI, dtQ, dtU, dtV, drQ, drU, drV) of
// the seven optical depths: the chain sum of src/rtesolver.f90:922-1000
// evaluated as one directional derivative.  lambda1 = x and lambda2 = y are
// differentiated through the larger root and x*y = |eta.rho| (no
// cancellation); theta = 0 and the reference's DAUX guards give zero.
__device__ __forceinline__ void evol_dir(const EvolSt& s, const EvolW& v, const float dt[7], float out[4]) {
  const float deQ = dt[1], deU = dt[2], deV = dt[3], drQ = dt[4], drU = dt[5], drV = dt[6];
  const float ede = s.tQ * deQ + s.tU * deU + s.tV * deV;
  const float rdr = s.rQ * drQ + s.rU * drU + s.rV * drV;
  const float der = s.rQ * deQ + s.rU * deU + s.rV * deV + s.tQ * drQ + s.tU * drU + s.tV * drV;
  // the layer's reciprocals come with its state: 1/R = 2 (0.5/R) exactly,
  // 0.5/root = 0.5 (1/root) exactly; the quotients by the root are products
  const float iR = 2.0f * s.it;
  const float dth = (s.d * (ede - rdr) + 2.0f * s.er * der) * iR;   // d theta
  float dx = 0.0f, dy = 0.0f;
  if (s.d >= 0.0f) {
    if (s.x > 0.0f) {
      dx = (0.5f * dth + ede - rdr) * (0.5f * s.iv);
      dy = (s.sg * der - s.y * dx) * s.iv;
    }
  } else if (s.y > 0.0f) {
    dy = (0.5f * dth - ede + rdr) * (0.5f * s.iv);
    dx = (s.sg * der - s.x * dy) * s.iv;
  }
  float Xd[4], Yd[4], M4d[4];
  xy_apply(deQ, deU, deV, drQ, drU, drV, v.w, Xd, Yd);
  {
    // d(raw M4) w: product rule on m4raw_apply
    const float dh = ede + rdr;
    const float cQ = (deU * s.rV - deV * s.rU) + (s.tU * drV - s.tV * drU);
    const float cU = (deV * s.rQ - deQ * s.rV) + (s.tV * drQ - s.tQ * drV);
    const float cV = (deQ * s.rU - deU * s.rQ) + (s.tQ * drU - s.tU * drQ);
    const float* w = v.w;
    const float ew = s.tQ * w[1] + s.tU * w[2] + s.tV * w[3], rw = s.rQ * w[1] + s.rU * w[2] + s.rV * w[3];
    const float dew = deQ * w[1] + deU * w[2] + deV * w[3], drw = drQ * w[1] + drU * w[2] + drV * w[3];
    M4d[0] = dh * w[0] + (cQ * w[1] + cU * w[2] + cV * w[3]);
    M4d[1] = -cQ * w[0] + deQ * ew + s.tQ * dew + drQ * rw + s.rQ * drw - dh * w[1];
    M4d[2] = -cU * w[0] + deU * ew + s.tU * dew + drU * rw + s.rU * drw - dh * w[2];
    M4d[3] = -cV * w[0] + deV * ew + s.tV * dew + drV * rw + s.rV * drw - dh * w[3];
  }
  const float a1 = 0.5f * (s.sh * dx - s.s2v * dy), a3 = -s.c2v * dy, a5 = -s.ch * dx;
  const float a7 = 0.5f * (s.sh * dx + s.s2v * dy);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    // d(M/theta) w = (-dtheta M w + d(raw M) w) / theta
    const float dM2 = (-dth * v.M2w[i] + (dy * v.Xw[i] + s.y * Xd[i] + s.sg * (dx * v.Yw[i] + s.x * Yd[i]))) * s.it;
    const float dM3 = (-dth * v.M3w[i] + (dx * v.Xw[i] + s.x * Xd[i] - s.sg * (dy * v.Yw[i] + s.y * Yd[i]))) * s.it;
    const float dM4 = (-dth * v.M4w[i] + 2.0f * M4d[i]) * s.it;
    const float inner = a1 * v.w[i] + a3 * v.M2w[i] - s.s2v * dM2 + a5 * v.M3w[i] - s.sh * dM3 + a7 * v.M4w[i] +
                        s.Qm * dM4;
    out[i] = s.E * inner - dt[0] * v.Ow[i];
  }
}

}  // namespace fzd
