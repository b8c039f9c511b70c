// firtez-dz B200: kernels and C-ABI of the Stokes synthesis path.
//
// Data flow of one fz_forward call (all on one stream):
//   k_chem   one warp per column, FP64: (optional) hydrostatic RK4 from the top,
//            chemical equilibrium per height, continuum/line opacity, damping,
//            Doppler widths and field geometry -> a per-column "opacity slab"
//            (nz rows of SW floats) in scratch memory, plus the updated model
//            (rho, Pe, mu, log tau5, Pg) like FORWARD1D writes it back.
//   k_synth  one CTA per column, one thread per wavelength, FP32: stages the
//            slab in shared memory, walks the heights bottom -> top evaluating
//            the Zeeman-split Voigt/Faraday profiles, the 4x4 evolution
//            operator and the formal-solution recurrence, writes RSYN1D.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/fz_b200.h"
#include "fz_host.h"
#include "fz_physics.cuh"

using namespace fzd;

namespace {

constexpr int MAXREG = 8;
constexpr int MAXLU = 16;     // lines used by the regions (main + blends)
constexpr int MAXCOMP = 256;  // Zeeman components of all used lines
constexpr int MAXNUMW = 1024;
constexpr int MAXNZ = 1024;

// Per-context constants read by the kernels (global memory, one copy per ctx).
struct DevParams {
  int nz, numw, nreg, nlu, sw;
  int reg_p0[MAXREG], reg_nw[MAXREG], reg_nb[MAXREG], reg_lb[MAXREG];
  double reg_l0[MAXREG];   // central wavelength of the region's main line [A]
  LineP lu[MAXLU];         // used lines in region order
  int lu_nc[MAXLU], lu_c0[MAXLU];
  float comp_shift[MAXCOMP], comp_str[MAXCOMP];
  int comp_type[MAXCOMP];
  double matom_h, matom_he, abund_he;
};

// Per-wavelength constants.
struct LamP {
  float wave;   // [mA] offset of the grid point
  float c1;     // 2 h c^2 / lambda^5
  float c2;     // h c / (lambda k)
  int reg;
};

// slab row layout
__host__ __device__ inline int slab_w(int nreg, int nlu) {
  const int w = 2 + nreg + 6 + 4 * nlu;
  return (w + 3) & ~3;
}
__host__ __device__ inline int slab_geo(int nreg) { return 2 + nreg; }
__host__ __device__ inline int slab_line(int nreg) { return 2 + nreg + 6; }

// ------------------------------------------------------------------ k_chem
__device__ __forceinline__ float mget(const float* m, int nz, int p, int k) { return m[p * nz + k]; }

// Per-height quantities of the slab (lanes split the work).
__device__ void fill_row(const DevParams& P, const Consts& K, float* row, int lane, float T, double nhyd,
                         double nelec, double dz, float bx, float by, float bz, float vz, float* kc5_out) {
  if (lane == 0) {
    double kc5 = opac_continuum(T, 5000.0, nelec, nhyd);
    kc5 = kc5 / nhyd * (1.0 / MAMU);
    row[0] = T;
    row[1] = (kc5 < KC5THRESHOLD) ? 0.0f : 1.0f;
    *kc5_out = (float)kc5;
  } else if (lane <= P.nreg) {
    const int r = lane - 1;
    const double kc = opac_continuum(T, P.reg_l0[r], nelec, nhyd);
    row[2 + r] = (float)(kc * dz);
  } else if (lane >= 9 && lane < 9 + P.nlu) {   // regions use lanes 1..8, lines 9..24
    const int b = lane - 9;
    const LineP& L = P.lu[b];
    const double klin = opac_line(L, T, nelec, nhyd, K);
    const double damp = get_damping(L, nhyd, T, K, P.matom_h, P.matom_he, P.abund_he);
    const double vdop = sqrt(2.0 * KBOL * (double)T / (L.matom * MAMU));
    const double dldop = 1e3 * (vdop * L.l0 / LIGHT);
    const double dlv = -1e3 * L.l0 * (double)vz / LIGHT;
    float* q = row + slab_line(P.nreg) + 4 * b;
    q[0] = (float)(klin * dz);
    q[1] = (float)damp;
    q[2] = (float)(1.0 / dldop);
    q[3] = (float)(dlv - L.wdif);
  } else if (lane == 31) {
    // field geometry, src/absorption_matrix.f90:919-991
    const double x = bx, y = by, z = bz;
    const double x2 = pow(x, 2.0), y2 = pow(y, 2.0), z2 = pow(z, 2.0);
    const double b2 = x2 + y2 + z2, b = sqrt(b2);
    double cosg = 0, cgf = 1, sgf = 1, c2p = 0, s2p = 0;
    if (b > 0) {
      cosg = z / b;
      cgf = 1 + z2 / b2;
      sgf = 1 - z2 / b2;
    }
    if (x != 0 || y != 0) {
      c2p = (x2 - y2) / (x2 + y2);
      s2p = 2. * x * y / (x2 + y2);
    }
    float* g = row + slab_geo(P.nreg);
    g[0] = (float)(0.25 * cgf);
    g[1] = (float)(0.5 * sgf);
    g[2] = (float)(sgf * c2p);
    g[3] = (float)(sgf * s2p);
    g[4] = (float)(0.5 * cosg);
    g[5] = (float)b;
  }
}

__device__ __forceinline__ double layer_dz(const float* m, int nz, int k) {
  // DELTAZ of EVOL_OPERATOR, src/rtesolver.f90:439-443 (z in km)
  return (k == nz - 1) ? 1e5 * fabs((double)mget(m, nz, 12, k) - (double)mget(m, nz, 12, k - 1))
                       : 1e5 * fabs((double)mget(m, nz, 12, k + 1) - (double)mget(m, nz, 12, k));
}

template <bool HE>
__global__ void __launch_bounds__(128) k_chem(const DevParams* __restrict__ Pg, const Consts* __restrict__ Kg,
                                              int ncol, const float* model, float* mout,
                                              float* __restrict__ slab, int* __restrict__ status) {
  extern __shared__ float sm_chem[];
  __shared__ Consts K;
  __shared__ DevParams P;
  {
    const int* src = reinterpret_cast<const int*>(Kg);
    int* dst = reinterpret_cast<int*>(&K);
    for (int i = threadIdx.x; i < (int)(sizeof(Consts) / 4); i += blockDim.x) dst[i] = src[i];
    const int* s2 = reinterpret_cast<const int*>(Pg);
    int* d2 = reinterpret_cast<int*>(&P);
    for (int i = threadIdx.x; i < (int)(sizeof(DevParams) / 4); i += blockDim.x) d2[i] = s2[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int col = blockIdx.x * (blockDim.x >> 5) + wib;
  if (col >= ncol) return;
  const int nz = P.nz, sw = P.sw;
  float* kc5s = sm_chem + wib * 2 * nz;   // per warp: kc5 (REAL) and rho
  float* rhos = kc5s + nz;
  const float* m = model + (size_t)col * 13 * nz;
  float* mo = mout + (size_t)col * 13 * nz;
  float* sl = slab + (size_t)col * nz * sw;
  if (mo != m)
    for (int i = lane; i < 13 * nz; i += 32) mo[i] = m[i];
  __syncwarp();
  int st = 0;
  if (!HE) {
    double nelec = 0.0;
    WarpSaha w;
    for (int k = 0; k < nz; ++k) {
      const float T = mget(m, nz, 0, k);
      saha_prepare(w, (double)T, K, lane);
      const RhoOut r = get_rho_warp(w, (double)mget(m, nz, 1, k), nelec, K, lane);
      st |= r.status;
      if (lane == 0) {
        const float rho = (float)r.dens;
        mo[2 * nz + k] = rho;
        mo[3 * nz + k] = (float)r.pelec;
        mo[4 * nz + k] = (float)r.molecw;
        rhos[k] = rho;
      }
      fill_row(P, K, sl + (size_t)k * sw, lane, T, r.nhyd, nelec, layer_dz(m, nz, k), mget(m, nz, 5, k),
               mget(m, nz, 6, k), mget(m, nz, 7, k), mget(m, nz, 10, k), &kc5s[k]);
    }
  } else {
    // RK4_INTEGRATION_LOG, src/hydrostatic_tools.f90:150-222, RK4_LOG :350-396
    const int top = nz - 1;
    double nelec = (double)mget(m, nz, 3, top) / KBOL / (double)mget(m, nz, 0, top);
    double t0 = (double)mget(m, nz, 12, top) * 1000.0 * 100.0;
    double u0 = log((double)mget(m, nz, 1, top));
    WarpSaha s0, sm, s1;
    saha_prepare(s0, (double)mget(m, nz, 0, top), K, lane);
    auto emit = [&](int k, double pg8, const RhoOut& r) {
      const float T = mget(m, nz, 0, k);
      const float pel = (float)r.pelec;
      if (lane == 0) {
        mo[1 * nz + k] = (float)exp(pg8);
        mo[2 * nz + k] = (float)r.dens;
        mo[3 * nz + k] = pel;
        mo[4 * nz + k] = (float)r.molecw;
        rhos[k] = (float)r.dens;
      }
      const double vnelec = (double)pel / KBOL / (double)T;   // src/forward.f90:900
      fill_row(P, K, sl + (size_t)k * sw, lane, T, r.nhyd, vnelec, layer_dz(m, nz, k), mget(m, nz, 5, k),
               mget(m, nz, 6, k), mget(m, nz, 7, k), mget(m, nz, 10, k), &kc5s[k]);
    };
    {
      const RhoOut r = get_rho_warp(s0, exp(u0), nelec, K, lane);
      st |= r.status;
      emit(top, u0, r);
    }
    for (int k = nz - 2; k >= 0; --k) {
      const double dz = ((double)mget(m, nz, 12, k) - (double)mget(m, nz, 12, k + 1)) * 1000.0 * 100.0;
      const double t1 = t0 + dz;
      const double tm0 = (double)mget(m, nz, 0, k + 1), tm1 = (double)mget(m, nz, 0, k);
      RhoOut q = get_rho_warp(s0, exp(u0), nelec, K, lane);
      st |= q.status;
      const double k1 = (-q.molecw * MAMU * GRAV / (KBOL * tm0)) * dz;
      const double it1 = t0 + dz / 2.0;
      const double iy1 = u0 + k1 / 2.0;
      const double tem = tm0 / dz * (t0 + dz - it1) + tm1 / dz * (it1 - t0);
      saha_prepare(sm, tem, K, lane);
      q = get_rho_warp(sm, exp(iy1), nelec, K, lane);
      st |= q.status;
      const double k2 = (-q.molecw * MAMU * GRAV / (KBOL * tem)) * dz;
      const double iy2 = u0 + k2 / 2.0;
      q = get_rho_warp(sm, exp(iy2), nelec, K, lane);
      st |= q.status;
      const double k3 = (-q.molecw * MAMU * GRAV / (KBOL * tem)) * dz;
      const double iy3 = u0 + k3;
      saha_prepare(s1, tm1, K, lane);
      q = get_rho_warp(s1, exp(iy3), nelec, K, lane);
      st |= q.status;
      const double k4 = (-q.molecw * MAMU * GRAV / (KBOL * tm1)) * dz;
      const double u1 = u0 + 1.0 / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4);
      q = get_rho_warp(s1, exp(u1), nelec, K, lane);
      st |= q.status;
      emit(k, u1, q);
      u0 = u1;
      t0 = t1;
      s0 = s1;
    }
  }
  __syncwarp();
  // log tau5 from the top, src/forward.f90:1000-1006 (REAL*4 accumulation)
  if (lane == 0) {
    float tau = 1e-9f;
    mo[11 * nz + nz - 1] = log10f(tau);
    for (int k = nz - 2; k >= 0; --k) {
      const float a = (kc5s[k] * rhos[k] + kc5s[k + 1] * rhos[k + 1]) / 2.0f;
      const double b = ((double)mget(m, nz, 12, k + 1) - (double)mget(m, nz, 12, k)) * 1000.0 * 100.0;
      tau = (float)((double)tau + (double)a * b);
      mo[11 * nz + k] = log10f(tau);
    }
    if (status) status[col] = st;
  }
}

// ----------------------------------------------------------------- k_synth
__global__ void __launch_bounds__(MAXNUMW) k_synth(const DevParams* __restrict__ Pg, const LamP* __restrict__ lam,
                                                   const float* __restrict__ gain, int ncol,
                                                   const float* __restrict__ slab, double* __restrict__ syn,
                                                   int* __restrict__ status) {
  extern __shared__ float4 sm_synth4[];
  float* sm = reinterpret_cast<float*>(sm_synth4);
  __shared__ DevParams P;
  {
    const int* s2 = reinterpret_cast<const int*>(Pg);
    int* d2 = reinterpret_cast<int*>(&P);
    for (int i = threadIdx.x; i < (int)(sizeof(DevParams) / 4); i += blockDim.x) d2[i] = s2[i];
  }
  const int col = blockIdx.x;
  const int nz = Pg->nz, sw = Pg->sw;
  // stage the column's slab (nz*sw floats, 16-byte rows) in shared memory
  {
    const float4* src = reinterpret_cast<const float4*>(slab + (size_t)col * nz * sw);
    const int n4 = nz * sw / 4;
    for (int i = threadIdx.x; i < n4; i += blockDim.x) sm_synth4[i] = __ldg(src + i);
  }
  __syncthreads();
  const int l = threadIdx.x;
  if (l >= P.numw) return;
  const LamP lp = lam[l];
  const int r = lp.reg;
  const int nb = P.reg_nb[r], lb = P.reg_lb[r];
  const int goff = slab_geo(P.nreg), loff = slab_line(P.nreg);
  float I0 = 0.f, I1 = 0.f, I2 = 0.f, I3 = 0.f;
  int bad = 0;
  for (int k = 0; k < nz; ++k) {
    const float* row = sm + k * sw;
    const float T = row[0];
    const float S = lp.c1 / expm1f(lp.c2 / T);
    if (k == 0 || row[1] != 0.0f) {   // SET_BOUNDARY, src/rtesolver.f90:1134-1147
      I0 = S;
      I1 = I2 = I3 = 0.f;
      continue;
    }
    const float g1 = row[goff], g2 = row[goff + 1], g3 = row[goff + 2], g4 = row[goff + 3], g5 = row[goff + 4],
                B = row[goff + 5];
    float tI = row[2 + r], tQ = 0.f, tU = 0.f, tV = 0.f, rQ = 0.f, rU = 0.f, rV = 0.f;
    for (int b = 0; b < nb; ++b) {
      const float* q = row + loff + 4 * (lb + b);
      const float kldz = q[0], a = q[1], idd = q[2];
      const float x0 = lp.wave + q[3];
      float h0 = 0.f, h1 = 0.f, h2 = 0.f, f0 = 0.f, f1 = 0.f, f2 = 0.f;
      const int c0 = P.lu_c0[lb + b], nc = P.lu_nc[lb + b];
      for (int c = c0; c < c0 + nc; ++c) {
        const float u = (x0 + P.comp_shift[c] * B) * idd;
        float h, f;
        voigt_f32(a, u, h, f);
        const float s = P.comp_str[c];
        const int ty = P.comp_type[c];
        if (ty < 0) {
          h0 = fmaf(s, h, h0);
          f0 = fmaf(s, f, f0);
        } else if (ty == 0) {
          h1 = fmaf(s, h, h1);
          f1 = fmaf(s, f, f1);
        } else {
          h2 = fmaf(s, h, h2);
          f2 = fmaf(s, f, f2);
        }
      }
      const float hs = h0 + h2, fs = f0 + f2;
      const float hl = 0.5f * h1 - 0.25f * hs, fl = 0.5f * f1 - 0.25f * fs;
      tI = fmaf(kldz, g1 * hs + g2 * h1, tI);
      tQ = fmaf(kldz, g3 * hl, tQ);
      tU = fmaf(kldz, g4 * hl, tU);
      tV = fmaf(kldz, g5 * (h0 - h2), tV);
      rQ = fmaf(kldz, g3 * fl, rQ);
      rU = fmaf(kldz, g4 * fl, rU);
      rV = fmaf(kldz, g5 * (f0 - f2), rV);
    }
    float O[16];
    if (!(isfinite(tI) && isfinite(tQ) && isfinite(tU) && isfinite(tV) && isfinite(rQ) && isfinite(rU) &&
          isfinite(rV))) {
      bad = 1;   // the reference replaces a non-finite matrix by the identity
#pragma unroll
      for (int i = 0; i < 16; ++i) O[i] = (i % 5 == 0) ? 1.f : 0.f;
    } else {
      evol_f32(tI, tQ, tU, tV, rQ, rU, rV, O);
    }
    // I_k = (1 - O) S + O I_{k-1}, src/rtesolver.f90:163-187
    const float n0 = fmaf(1.0f - O[0], S, fmaf(O[0], I0, fmaf(O[1], I1, fmaf(O[2], I2, O[3] * I3))));
    const float n1 = fmaf(-O[4], S, fmaf(O[4], I0, fmaf(O[5], I1, fmaf(O[6], I2, O[7] * I3))));
    const float n2 = fmaf(-O[8], S, fmaf(O[8], I0, fmaf(O[9], I1, fmaf(O[10], I2, O[11] * I3))));
    const float n3 = fmaf(-O[12], S, fmaf(O[12], I0, fmaf(O[13], I1, fmaf(O[14], I2, O[15] * I3))));
    I0 = n0;
    I1 = n1;
    I2 = n2;
    I3 = n3;
  }
  // CALCULATE_EQUIVALENT_SYN1D: x GAIN, Stokes-major
  const int nw = P.numw;
  double* o = syn + (size_t)col * 4 * nw;
  o[0 * nw + l] = (double)I0 * (double)gain[4 * l + 0];
  o[1 * nw + l] = (double)I1 * (double)gain[4 * l + 1];
  o[2 * nw + l] = (double)I2 * (double)gain[4 * l + 2];
  o[3 * nw + l] = (double)I3 * (double)gain[4 * l + 3];
  if (!(isfinite(I0) && isfinite(I1) && isfinite(I2) && isfinite(I3))) bad = 1;
  if (status && __any_sync(__activemask(), bad) && (l & 31) == 0) atomicOr(&status[col], FZ_NAN);
}

// ------------------------------------------------------------------ k_gain
// HSRA continuum normalisation, src/normalization.f90:696-754: one block;
// warp 0 runs the chemistry of the 387 layers (nelec chain), then every
// thread integrates its wavelengths through the continuum-only atmosphere
// with the reference's REAL*4 rounding of the intermediate intensities.
__global__ void k_gain(const DevParams* __restrict__ Pg, const Consts* __restrict__ Kg,
                       const double* __restrict__ lam_l /* (numw) full wavelength [A] */, float* gain,
                       int* status) {
  extern __shared__ double sm_gain[];   // (387 x nreg) continuum opacities
  const DevParams& P = *Pg;
  const Consts& K = *Kg;
  const int N = FZ_HSRA_LEN;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    double nelec = 0.0;
    WarpSaha w;
    int st = 0;
    for (int k = 0; k < N; ++k) {
      const float T = fz_tab_hsra_tem[k];
      saha_prepare(w, (double)T, K, lane);
      const RhoOut r = get_rho_warp(w, (double)fz_tab_hsra_pg[k], nelec, K, lane);
      st |= r.status;
      if (lane < P.nreg) sm_gain[k * P.nreg + lane] = opac_continuum(T, P.reg_l0[lane], nelec, r.nhyd);
    }
    if (lane == 0 && status) *status = st;
  }
  __syncthreads();
  for (int l = threadIdx.x; l < P.numw; l += blockDim.x) {
    int reg = 0;
    for (int q = 0; q < P.nreg; ++q)
      if (l >= P.reg_p0[q]) reg = q;
    const double w = lam_l[l] * 1e-8;
    double syn = 0.0;
    for (int k = 0; k < N; ++k) {
      const double T = (double)fz_tab_hsra_tem[k];
      const double S = (double)(float)(2.0 * HPLA * pow(LIGHT, 2.0) / pow(w, 5.0) *
                                       (1.0 / (exp(HPLA * LIGHT / (w * KBOL * T)) - 1.0)));
      if (k == 0) {
        syn = S;
        continue;
      }
      double ei = sm_gain[k * P.nreg + reg];
      const bool imat = (ei == ei + 1.0);
      if (imat) ei = 1e15;
      const double dz = (k == N - 1) ? 1e5 * (double)fabsf(fz_tab_hsra_z[k] - fz_tab_hsra_z[k - 1])
                                     : 1e5 * (double)fabsf(fz_tab_hsra_z[k + 1] - fz_tab_hsra_z[k]);
      double ev = exp(-ei * dz) * (0.5 * (1.0 + 1.0) * 1.0);
      if (imat) ev = 1.0;
      syn = (double)(float)((1.0 - ev) * S + ev * syn);
    }
    const float g = (float)(1.0 / syn);
    gain[4 * l + 0] = g;
    gain[4 * l + 1] = g;
    gain[4 * l + 2] = g;
    gain[4 * l + 3] = -g;   // V sign convention, :743
  }
}

// --------------------------------------------------- FP32 peak probe
// 8 independent FMA chains per thread, 4096 FMAs each, register resident.
__global__ void k_fp32_peak(float* out, int iters, float s) {
  float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
  float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
  const float m = 0.9999999f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 64; ++j) {
      a0 = fmaf(a0, m, s); a1 = fmaf(a1, m, s); a2 = fmaf(a2, m, s); a3 = fmaf(a3, m, s);
      a4 = fmaf(a4, m, s); a5 = fmaf(a5, m, s); a6 = fmaf(a6, m, s); a7 = fmaf(a7, m, s);
    }
  }
  const float r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (r == 1234.5f) out[0] = r;   // keeps the chains live
}

// ------------------------------------------------------------------ context
void host_consts(Consts& K) {
  K.csaha1 = std::pow(HPLA, 3.0) / std::pow(2.0 * DPI * MELE * KBOL, 3.0 / 2.0);
  K.csaha2 = EVOLT / KBOL;
  K.rbohr = std::pow(HPLA, 2.0) / (4.0 * std::pow(DPI, 2.0) * MELE * std::pow(QELE, 2.0));
  K.deno_sa = 0.0;
  K.deno_sam = 0.0;
  static const double ab[FZ_NELEM] = {
#include "fz_abund.inc"
  };
  for (int i = 0; i < FZ_NELEM; ++i) {
    K.ab10[i] = std::pow(10.0, ab[i] - 12.0);
    K.deno_sa = K.deno_sa + K.ab10[i];
  }
  static const double mat[FZ_NELEM] = {
#include "fz_matom.inc"
  };
  for (int i = 0; i < FZ_NELEM; ++i) K.deno_sam = K.deno_sam + MAMU * mat[i] * K.ab10[i];
}

}  // namespace

struct fz_ctx {
  int device = 0;
  int nz = 0, numw = 0, nreg = 0, nlu = 0, sw = 0;
  std::vector<fz_line> lines;
  std::vector<fz_region> regs;
  std::vector<float> gain;   // (4, numw)
  DevParams hp{};
  DevParams* d_params = nullptr;
  Consts* d_consts = nullptr;
  LamP* d_lam = nullptr;
  float* d_gain = nullptr;
  // scratch (grown on demand)
  float* d_slab = nullptr;
  size_t slab_cols = 0;
  // staging for the host-buffer API
  float* d_model = nullptr;
  double* d_syn = nullptr;
  int* d_status = nullptr;
  size_t io_cols = 0;
  cudaStream_t stream = nullptr;
  // per-kernel profiling (pending event pairs are resolved on read)
  bool prof = false;
  struct Pending {
    int kernel;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  double prof_ms[2] = {0, 0};
  int prof_n[2] = {0, 0};
};

namespace {

int cuda_fail(cudaError_t e) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "fz_b200: CUDA error %s\n", cudaGetErrorString(e));
    return FZ_ERR_CUDA;
  }
  return 0;
}
#define FZ_CK(x)                              \
  do {                                        \
    int _rc = cuda_fail(x);                   \
    if (_rc) return _rc;                      \
  } while (0)

int ensure_slab(fz_ctx* c, int ncol) {
  if ((size_t)ncol <= c->slab_cols) return 0;
  if (c->d_slab) cudaFree(c->d_slab);
  c->d_slab = nullptr;
  c->slab_cols = 0;
  FZ_CK(cudaMalloc(&c->d_slab, (size_t)ncol * c->nz * c->sw * sizeof(float)));
  c->slab_cols = ncol;
  return 0;
}

struct ProfScope {
  fz_ctx* c;
  int kernel;
  cudaStream_t s;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(fz_ctx* c_, int k, cudaStream_t s_) : c(c_), kernel(k), s(s_) {
    if (!c->prof) return;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
  }
  ~ProfScope() {
    if (!c->prof) return;
    cudaEventRecord(b, s);
    c->pending.push_back({kernel, a, b});
  }
};

int launch_forward(fz_ctx* c, int ncol, const float* d_model, int hydrostatic, double* d_syn, float* d_mout,
                   int* d_status, cudaStream_t s) {
  int rc = ensure_slab(c, ncol);
  if (rc) return rc;
  if (d_status) FZ_CK(cudaMemsetAsync(d_status, 0, ncol * sizeof(int), s));
  const int wpb = 4;
  const size_t smc = (size_t)wpb * 2 * c->nz * sizeof(float);
  const dim3 gc((ncol + wpb - 1) / wpb);
  {
    ProfScope ps(c, 0, s);
    if (hydrostatic)
      k_chem<true><<<gc, wpb * 32, smc, s>>>(c->d_params, c->d_consts, ncol, d_model, d_mout, c->d_slab, d_status);
    else
      k_chem<false><<<gc, wpb * 32, smc, s>>>(c->d_params, c->d_consts, ncol, d_model, d_mout, c->d_slab, d_status);
  }
  FZ_CK(cudaGetLastError());
  const int threads = (c->numw + 31) & ~31;
  const size_t sms = (size_t)c->nz * c->sw * sizeof(float);
  {
    ProfScope ps(c, 1, s);
    k_synth<<<ncol, threads, sms, s>>>(c->d_params, c->d_lam, c->d_gain, ncol, c->d_slab, d_syn, d_status);
  }
  FZ_CK(cudaGetLastError());
  return 0;
}

}  // namespace

extern "C" {

int fz_version(void) { return 100; }

const char* fz_strerror(int code) {
  switch (code) {
    case 0: return "ok";
    case FZ_ERR_ARG: return "invalid argument";
    case FZ_ERR_CUDA: return "CUDA error";
    case FZ_ERR_NOMEM: return "out of memory";
    case FZ_ERR_PARSE: return "line database parse error";
    case FZ_ERR_LIMIT: return "size limit exceeded";
    case FZ_ERR_STATE: return "invalid state";
  }
  return "unknown error";
}

int fz_lines_parse(const char* text, fz_line* out, int maxn) { return fzh_lines_parse(text, out, maxn); }

int fz_numw(const fz_ctx* c) { return c ? c->numw : FZ_ERR_ARG; }

int fz_create(fz_ctx** out, const fz_line* lines, int nlines, const fz_region* regs, int nreg, int nz,
              const float* gain, int device) {
  if (!out || !lines || nlines <= 0 || nlines > FZ_MAXLINES || !regs || nreg <= 0 || nreg > MAXREG || nz < 2 ||
      nz > MAXNZ)
    return FZ_ERR_ARG;
  *out = nullptr;
  fz_ctx* c = new (std::nothrow) fz_ctx;
  if (!c) return FZ_ERR_NOMEM;
  c->device = device;
  c->nz = nz;
  c->nreg = nreg;
  c->lines.assign(lines, lines + nlines);
  c->regs.assign(regs, regs + nreg);
  DevParams& P = c->hp;
  std::memset(&P, 0, sizeof(P));
  int numw = 0, nlu = 0, ncomp = 0;
  std::vector<LamP> lam;
  std::vector<double> lam_l;
  for (int r = 0; r < nreg; ++r) {
    const fz_region& R = regs[r];
    if (R.nblend < 1 || R.nblend > FZ_MAXBLEND || R.numwave < 1) {
      delete c;
      return FZ_ERR_ARG;
    }
    P.reg_p0[r] = numw;
    P.reg_nw[r] = R.numwave;
    P.reg_nb[r] = R.nblend;
    P.reg_lb[r] = nlu;
    const fz_line& main = lines[R.line[0]];
    P.reg_l0[r] = main.l0;
    for (int b = 0; b < R.nblend; ++b) {
      if (R.line[b] < 0 || R.line[b] >= nlines || nlu >= MAXLU) {
        delete c;
        return nlu >= MAXLU ? FZ_ERR_LIMIT : FZ_ERR_ARG;
      }
      const fz_line& L = lines[R.line[b]];
      LineP& q = P.lu[nlu];
      q.l0 = L.l0;
      q.loggf = L.loggf;
      q.eplow = L.eplow;
      q.alpha = L.alpha;
      q.sigma = L.sigma;
      q.zn = L.zn;
      q.ion = L.ion;
      q.wdif = b == 0 ? 0.0 : R.wdif[b];
      std::vector<double> sh, stg;
      std::vector<int> ty;
      const int n = fzh_zeeman(L, sh, stg, ty);
      if (n < 0 || ncomp + n > MAXCOMP) {
        delete c;
        return n < 0 ? FZ_ERR_ARG : FZ_ERR_LIMIT;
      }
      P.lu_c0[nlu] = ncomp;
      P.lu_nc[nlu] = n;
      for (int i = 0; i < n; ++i) {
        P.comp_shift[ncomp + i] = (float)sh[i];
        P.comp_str[ncomp + i] = (float)stg[i];
        P.comp_type[ncomp + i] = ty[i];
      }
      ncomp += n;
      ++nlu;
    }
    for (int j = 0; j < R.numwave; ++j) {
      const double wv = R.wave_ini + R.dlambda * (double)j;   // WAVE_INIT
      const double w = (main.l0 + wv / 1.0e3) * 1e-8;        // SOURCE_FUNCTION [cm]
      LamP p;
      p.wave = (float)wv;
      p.c1 = (float)(2.0 * HPLA * std::pow(LIGHT, 2.0) / std::pow(w, 5.0));
      p.c2 = (float)(HPLA * LIGHT / (w * KBOL));
      p.reg = r;
      lam.push_back(p);
      lam_l.push_back(main.l0 + wv / 1.0e3);
    }
    numw += R.numwave;
  }
  if (numw > MAXNUMW) {
    delete c;
    return FZ_ERR_LIMIT;
  }
  c->numw = numw;
  c->nlu = nlu;
  c->sw = slab_w(nreg, nlu);
  P.nz = nz;
  P.numw = numw;
  P.nreg = nreg;
  P.nlu = nlu;
  P.sw = c->sw;
  Consts K;
  host_consts(K);
  {
    static const double mat[FZ_NELEM] = {
#include "fz_matom.inc"
    };
    static const double ab[FZ_NELEM] = {
#include "fz_abund.inc"
    };
    for (int b = 0; b < nlu; ++b) {
      P.lu[b].matom = mat[P.lu[b].zn - 1];
      P.lu[b].abund = ab[P.lu[b].zn - 1];
    }
    P.matom_h = mat[0];
    P.matom_he = mat[1];
    P.abund_he = ab[1];
  }
  int rc = 0;
  auto fail = [&](int code) {
    fz_destroy(c);
    return code;
  };
  if ((rc = cuda_fail(cudaSetDevice(device)))) return fail(rc);
  if ((rc = cuda_fail(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)))) return fail(rc);
  if ((rc = cuda_fail(cudaMalloc(&c->d_params, sizeof(DevParams))))) return fail(rc);
  if ((rc = cuda_fail(cudaMalloc(&c->d_consts, sizeof(Consts))))) return fail(rc);
  if ((rc = cuda_fail(cudaMalloc(&c->d_lam, numw * sizeof(LamP))))) return fail(rc);
  if ((rc = cuda_fail(cudaMalloc(&c->d_gain, 4 * numw * sizeof(float))))) return fail(rc);
  if ((rc = cuda_fail(cudaMemcpy(c->d_params, &P, sizeof(P), cudaMemcpyHostToDevice)))) return fail(rc);
  if ((rc = cuda_fail(cudaMemcpy(c->d_consts, &K, sizeof(K), cudaMemcpyHostToDevice)))) return fail(rc);
  if ((rc = cuda_fail(cudaMemcpy(c->d_lam, lam.data(), numw * sizeof(LamP), cudaMemcpyHostToDevice))))
    return fail(rc);
  c->gain.assign(4 * numw, 0.0f);
  if (gain) {
    std::memcpy(c->gain.data(), gain, 4 * numw * sizeof(float));
    if ((rc = cuda_fail(cudaMemcpy(c->d_gain, gain, 4 * numw * sizeof(float), cudaMemcpyHostToDevice))))
      return fail(rc);
  } else {
    double* d_l = nullptr;
    int* d_st = nullptr;
    if ((rc = cuda_fail(cudaMalloc(&d_l, numw * sizeof(double))))) return fail(rc);
    if ((rc = cuda_fail(cudaMalloc(&d_st, sizeof(int))))) {
      cudaFree(d_l);
      return fail(rc);
    }
    cudaMemcpy(d_l, lam_l.data(), numw * sizeof(double), cudaMemcpyHostToDevice);
    k_gain<<<1, 256, FZ_HSRA_LEN * nreg * sizeof(double), c->stream>>>(c->d_params, c->d_consts, d_l, c->d_gain,
                                                                        d_st);
    rc = cuda_fail(cudaGetLastError());
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(c->stream));
    int st = 0;
    if (!rc) rc = cuda_fail(cudaMemcpy(&st, d_st, sizeof(int), cudaMemcpyDeviceToHost));
    if (!rc) rc = cuda_fail(cudaMemcpy(c->gain.data(), c->d_gain, 4 * numw * sizeof(float), cudaMemcpyDeviceToHost));
    cudaFree(d_l);
    cudaFree(d_st);
    if (rc) return fail(rc);
  }
  // opt in to large dynamic shared memory for the slab staging
  const int sms = nz * c->sw * (int)sizeof(float);
  if (sms > 48 * 1024) {
    if ((rc = cuda_fail(cudaFuncSetAttribute(k_synth, cudaFuncAttributeMaxDynamicSharedMemorySize, sms))))
      return fail(rc);
  }
  *out = c;
  return 0;
}

int fz_measure_fp32_peak(int device, double* tflops) {
  if (!tflops) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(device));
  int sms = 0;
  FZ_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  float* d = nullptr;
  FZ_CK(cudaMalloc(&d, sizeof(float)));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int threads = 512, blocks = sms * 4, iters = 64;
  k_fp32_peak<<<blocks, threads>>>(d, iters, 1e-7f);   // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(a);
    k_fp32_peak<<<blocks, threads>>>(d, iters, 1e-7f);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    best = t < best ? t : best;
  }
  const int rc = cuda_fail(cudaGetLastError());
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d);
  if (rc) return rc;
  const double fma = (double)blocks * threads * iters * 64 * 8;
  *tflops = 2.0 * fma / (best * 1e-3) / 1e12;
  return 0;
}

int fz_destroy(fz_ctx* c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->d_params);
  cudaFree(c->d_consts);
  cudaFree(c->d_lam);
  cudaFree(c->d_gain);
  cudaFree(c->d_slab);
  cudaFree(c->d_model);
  cudaFree(c->d_syn);
  cudaFree(c->d_status);
  for (auto& p : c->pending) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

int fz_profile_enable(fz_ctx* c, int on) {
  if (!c) return FZ_ERR_ARG;
  c->prof = on != 0;
  return 0;
}

int fz_profile_read(fz_ctx* c, double* ms, int* launches, int n) {
  if (!c) return FZ_ERR_ARG;
  for (auto& p : c->pending) {
    float t = 0.f;
    if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) {
      c->prof_ms[p.kernel] += t;
      c->prof_n[p.kernel] += 1;
    }
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  c->pending.clear();
  for (int i = 0; i < n && i < 2; ++i) {
    if (ms) ms[i] = c->prof_ms[i];
    if (launches) launches[i] = c->prof_n[i];
    c->prof_ms[i] = 0;
    c->prof_n[i] = 0;
  }
  return 2;
}

int fz_get_gain(fz_ctx* c, float* gain) {
  if (!c || !gain) return FZ_ERR_ARG;
  std::memcpy(gain, c->gain.data(), c->gain.size() * sizeof(float));
  return 0;
}

int fz_forward_device(fz_ctx* c, int ncol, const float* d_model, int hydrostatic, double* d_syn,
                      float* d_model_out, int* d_status, void* stream) {
  if (!c || ncol <= 0 || !d_model || !d_syn || !d_model_out) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  return launch_forward(c, ncol, d_model, hydrostatic, d_syn, d_model_out, d_status, (cudaStream_t)stream);
}

int fz_forward(fz_ctx* c, int ncol, const float* model, int hydrostatic, double* syn, float* model_out,
               int* status) {
  if (!c || ncol <= 0 || !model || !syn) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  if ((size_t)ncol > c->io_cols) {
    cudaFree(c->d_model);
    cudaFree(c->d_syn);
    cudaFree(c->d_status);
    c->d_model = nullptr;
    c->d_syn = nullptr;
    c->d_status = nullptr;
    c->io_cols = 0;
    FZ_CK(cudaMalloc(&c->d_model, (size_t)ncol * 13 * c->nz * sizeof(float)));
    FZ_CK(cudaMalloc(&c->d_syn, (size_t)ncol * 4 * c->numw * sizeof(double)));
    FZ_CK(cudaMalloc(&c->d_status, (size_t)ncol * sizeof(int)));
    c->io_cols = ncol;
  }
  cudaStream_t s = c->stream;
  const size_t mb = (size_t)ncol * 13 * c->nz * sizeof(float);
  FZ_CK(cudaMemcpyAsync(c->d_model, model, mb, cudaMemcpyHostToDevice, s));
  int rc = launch_forward(c, ncol, c->d_model, hydrostatic, c->d_syn, c->d_model, c->d_status, s);
  if (rc) return rc;
  FZ_CK(cudaMemcpyAsync(syn, c->d_syn, (size_t)ncol * 4 * c->numw * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (model_out) FZ_CK(cudaMemcpyAsync(model_out, c->d_model, mb, cudaMemcpyDeviceToHost, s));
  if (status) FZ_CK(cudaMemcpyAsync(status, c->d_status, ncol * sizeof(int), cudaMemcpyDeviceToHost, s));
  FZ_CK(cudaStreamSynchronize(s));
  return 0;
}

}  // extern "C"
