// firtez-dz B200: kernels and C-ABI of the Stokes synthesis path.
//
// Data flow of one fz_forward call (all on one stream):
//   k_chain  one warp per column, FP64, lanes over the 92 elements: the
//            sequential part of FORWARD1D -- the GET_RHO warm-start chain along
//            z and, in hydrostatic mode, the RK4 integration of ln Pg from the
//            top.  Writes (nH, ne) per height to scratch and rho, Pe, mu, Pg
//            into the output model.
//   k_opac   one thread per (column, height), FP64: continuum/line opacity,
//            damping, Doppler width, velocity shift and field geometry ->
//            the per-column "opacity slab" (nz rows of SW floats) in scratch.
//   k_synth  one CTA per column, one thread per wavelength, FP32: stages the
//            slab in shared memory, walks the heights bottom -> top evaluating
//            the Zeeman-split Voigt/Faraday profiles, the 4x4 evolution
//            operator and the formal-solution recurrence, writes RSYN1D; one
//            thread integrates log tau5.
#include <cuda_bf16.h>
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
#include "fz_rf.cuh"

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
  ContP cont[MAXREG + 1];   // continuum constants of each region's main line, then 5000 A
  LineP lu[MAXLU];          // used lines in region order
  int lu_nc[MAXLU], lu_c0[MAXLU];
  int lu_nt[MAXLU][3];      // components per type: sigma_red, pi, sigma_blue
  float lu_duv[MAXLU];      // -1e3 lambda0 / c: d u / d v_z = lu_duv / Doppler width [mA]
  float comp_shift[MAXCOMP], comp_str[MAXCOMP];
  int comp_type[MAXCOMP];
};

// Per-wavelength constants.
struct LamP {
  float wave;   // [mA] offset of the grid point
  float c1;     // 2 h c^2 / lambda^5
  float c2;     // h c / (lambda k)
  int reg;
};

// slab row layout: T, boundary flag, KC5 (REAL), rho (REAL), kc*dz per
// region, 6 field-geometry factors, 4 floats per used line
__host__ __device__ inline int slab_w(int nreg, int nlu) {
  const int w = 4 + nreg + 6 + 4 * nlu;
  return (w + 3) & ~3;
}
__host__ __device__ inline int slab_geo(int nreg) { return 4 + nreg; }
__host__ __device__ inline int slab_line(int nreg) { return 4 + nreg + 6; }

__device__ __forceinline__ float mget(const float* m, int nz, int p, int k) { return m[p * nz + k]; }

template <typename T>
__device__ __forceinline__ void copy_to_shared(T* dst, const T* src) {
  const int* s = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(T) / 4); i += blockDim.x) d[i] = s[i];
}

// ----------------------------------------------------------------- k_chain
// The temperature at the midpoint of an RK4 step of dz from height t0 (the
// linear interpolation of RK4_LOG, src/hydrostatic_tools.f90:377), written
// once for k_chain and k_saha so both round alike.
__device__ __forceinline__ double chain_tmid(double t0, double dz, double tm0, double tm1) {
  const double it1 = t0 + dz / 2.0;
  return tm0 / dz * (t0 + dz - it1) + tm1 / dz * (it1 - t0);
}

// One warp per column walks the heights sequentially: the GET_RHO warm-start
// chain (NELEC of one call seeds the next, src/forward.f90:914) and, in
// hydrostatic mode, the RK4 integration of ln Pg from the top
// (RK4_INTEGRATION_LOG, src/hydrostatic_tools.f90:150-222, RK4_LOG :350-396).
// Writes per height (nH, ne) as FORWARD1D uses them, and rho, Pe, mu (and
// Pg) into the output model.
//
// L lanes per column: 32 (a warp) or 16 (two columns per warp: each lane
// holds six elements, and every per-column scalar of the chain costs half
// the warp instructions).  At most 128 registers a thread (four blocks, 16
// warps per SM): the chain is bound by dependent FP64 latency, so resident
// warps count more than the few spilled values.
//
// PRE: the Saha factors of every temperature sample come precomputed from
// k_saha (rows sa of the columns [c0, c0 + cn) of the list), and the chain
// keeps only what is sequential: the GET_RHO iterations and the RK4 steps --
// half the latency of a column's chain, the form for small batches (an
// inversion's tail); on full batches the Saha work fills the stalls of the
// GET_RHO iterations and the plain form is faster.  gate > 0: run only when
// the column count is at most gate; gate < 0: only when it is above -gate (a
// captured launch over a device-side count takes the form that suits it).
template <bool HE, int L, bool PRE>
__global__ void __launch_bounds__(128, 4) k_chain(const Consts* __restrict__ Kg, const PFTable* __restrict__ tb, int ncol,
                                               int nz, const float* model, float* mout, double2* __restrict__ chem,
                                               int* __restrict__ status, const int* __restrict__ list = nullptr,
                                               const int* __restrict__ nlist = nullptr,
                                               const double2* __restrict__ sa = nullptr, int c0 = 0, int cn = 0,
                                               int gate = 0) {
  constexpr int NS = WarpSahaT<L>::NS;
  // listed columns (list[0, *nlist) of the ncol slots): a CTA past the end
  // of the list leaves before any work
  const int count = list ? *nlist : ncol;
  if ((gate > 0 && count > gate) || (gate < 0 && count <= -gate)) return;
  const int end = PRE ? min(count, c0 + cn) : count;
  const int first = PRE ? c0 : 0;
  if (first + (int)((blockIdx.x * (size_t)blockDim.x) / L) >= end) return;
  __shared__ Consts K;
  copy_to_shared(&K, Kg);
  __syncthreads();
  const int lane = threadIdx.x & (L - 1);
  const int g = first + (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) / L);
  if (g >= end) return;
  const int col = list ? list[g] : g;
  const int nsamp = HE ? 2 * nz - 1 : nz;
  const double2* rows = PRE ? sa + (size_t)(g - first) * nsamp * 96 : nullptr;
  const unsigned hyd = saha_hyd<L>(K, lane);
  const float* m = model + (size_t)col * 13 * nz;
  float* mo = mout + (size_t)col * 13 * nz;
  double2* ch = chem + (size_t)col * nz;
  if (mo != m)
    for (int i = lane; i < 13 * nz; i += L) mo[i] = m[i];
  __syncwarp(group_mask<L>());
  double ab[NS];
#pragma unroll
  for (int j = 0; j < NS; ++j) ab[j] = K.lane_elem[L * j + lane] >= 0 ? K.ab10[K.lane_elem[L * j + lane]] : 0.0;
  int st = 0;
  if (!HE) {
    double nelec = 0.0;
    WarpSahaT<L> w;
    for (int k = 0; k < nz; ++k) {
      if (PRE)
        saha_load(w, (double)mget(m, nz, 0, k), hyd, rows + (size_t)k * 96, lane);
      else
        saha_prepare(w, (double)mget(m, nz, 0, k), K, tb, lane);
      const RhoOut r = get_rho_warp(w, ab, (double)mget(m, nz, 1, k), nelec, K, lane);
      st |= r.status;
      if (lane == 0) {
        mo[2 * nz + k] = (float)r.dens;
        mo[3 * nz + k] = (float)r.pelec;
        mo[4 * nz + k] = (float)r.molecw;
        ch[k] = make_double2(r.nhyd, nelec);
      }
    }
  } else {
    const int top = nz - 1;
    double nelec = (double)mget(m, nz, 3, top) / KBOL / (double)mget(m, nz, 0, top);
    double t0 = (double)mget(m, nz, 12, top) * 1000.0 * 100.0;
    double u0 = log((double)mget(m, nz, 1, top));
    // One Saha buffer serves the whole integration: within a step the RK4
    // stages need T(k+1) (stage 1), the linear midpoint (stages 2, 3) and
    // T(k) (stage 4 and the final GET_RHO), and T(k) is the next step's T(k+1).
    WarpSahaT<L> w;
    if (PRE)
      saha_load(w, (double)mget(m, nz, 0, top), hyd, rows, lane);
    else
      saha_prepare(w, (double)mget(m, nz, 0, top), K, tb, lane);
    {
      const RhoOut r = get_rho_warp(w, ab, exp(u0), nelec, K, lane);
      st |= r.status;
      if (lane == 0) {
        const float pel = (float)r.pelec;
        mo[1 * nz + top] = (float)exp(u0);
        mo[2 * nz + top] = (float)r.dens;
        mo[3 * nz + top] = pel;
        mo[4 * nz + top] = (float)r.molecw;
        ch[top] = make_double2(r.nhyd, (double)pel / KBOL / (double)mget(m, nz, 0, top));
      }
    }
    for (int k = nz - 2; k >= 0; --k) {
      const double dz = ((double)mget(m, nz, 12, k) - (double)mget(m, nz, 12, k + 1)) * 1000.0 * 100.0;
      const double t1 = t0 + dz;
      const double tm0 = (double)mget(m, nz, 0, k + 1), tm1 = (double)mget(m, nz, 0, k);
      const double tmid = chain_tmid(t0, dz, tm0, tm1);
      const double2* srow = PRE ? rows + (size_t)(2 * (nz - 2 - k) + 1) * 96 : nullptr;   // the midpoint's row, then T(k)'s
      double kk[4] = {0.0, 0.0, 0.0, 0.0};
      double u1 = 0.0;
#pragma unroll 1
      for (int stg = 0; stg < 5; ++stg) {
        if (stg == 1 || stg == 3) {
          if (PRE)
            saha_load(w, stg == 1 ? tmid : tm1, hyd, stg == 1 ? srow : srow + 96, lane);
          else
            saha_prepare(w, stg == 1 ? tmid : tm1, K, tb, lane);
        }
        const double tem = stg == 0 ? tm0 : (stg < 3 ? tmid : tm1);
        const double y = stg == 0 ? u0 : (stg == 1 ? u0 + kk[0] / 2.0 : (stg == 2 ? u0 + kk[1] / 2.0 : (stg == 3 ? u0 + kk[2] : u1)));
        const RhoOut q = get_rho_warp(w, ab, exp(y), nelec, K, lane);
        st |= q.status;
        if (stg < 4) {
          const double d = (-q.molecw * MAMU * GRAV / (KBOL * tem)) * dz;
          kk[0] = stg == 0 ? d : kk[0];
          kk[1] = stg == 1 ? d : kk[1];
          kk[2] = stg == 2 ? d : kk[2];
          kk[3] = stg == 3 ? d : kk[3];
          if (stg == 3) u1 = u0 + 1.0 / 6.0 * (kk[0] + 2.0 * kk[1] + 2.0 * kk[2] + kk[3]);
        } else if (lane == 0) {
          const float pel = (float)q.pelec;
          mo[1 * nz + k] = (float)exp(u1);
          mo[2 * nz + k] = (float)q.dens;
          mo[3 * nz + k] = pel;
          mo[4 * nz + k] = (float)q.molecw;
          // FORWARD1D uses NELEC = PEL/KBOL/TEM from the REAL*4 model (src/forward.f90:900)
          ch[k] = make_double2(q.nhyd, (double)pel / KBOL / tm1);
        }
      }
      u0 = u1;
      t0 = t1;
    }
  }
  if (lane == 0 && status) status[col] = st;
}

// ------------------------------------------------------------------ k_saha
// The Saha factors of every temperature sample of k_chain's integration, for
// the listed columns [c0, c0 + cn): the samples are the model's T at each
// height and, with HE, the RK4 midpoint temperature of each step --
// functions of the model alone -- so this half of the chemistry's FP64 work
// leaves the sequential chain and runs with every (sample, element slot) in
// parallel, one CTA per column.  Row s of the i-th column of the chunk:
// sa[(i * nsamp + s) * 96 + slot] = (a1, a2) of the slot's element; samples
// (HE) 0 = T(top), 2j+1 = the midpoint of step j (height nz-2-j) and 2j+2 =
// T(nz-2-j); without HE, s = T(s).  A warp takes one sample at a time, lane
// l the slots l, l + 32 and l + 64 (its elements fixed for the whole
// column, so their table lines stay in L1); gridDim.y CTAs share a column's
// samples (small batches: latency).  gate > 0: run only when the column
// count is at most gate.
__host__ __device__ inline size_t saha_smem(int nz) {
  return (size_t)(2 * nz - 1) * (sizeof(double) + sizeof(SahaT)) + (size_t)2 * nz * sizeof(double);
}

template <bool HE>
__global__ void __launch_bounds__(256) k_saha(const Consts* __restrict__ Kg, const PFTable* __restrict__ tb,
                                              int ncol, int nz, const float* __restrict__ model,
                                              double2* __restrict__ sa, int c0, int cn,
                                              const int* __restrict__ list, const int* __restrict__ nlist,
                                              int gate) {
  extern __shared__ double sm_saha[];
  __shared__ Consts K;
  const int count = list ? *nlist : ncol;
  if (gate > 0 && count > gate) return;
  const int g = c0 + (int)blockIdx.x;
  if ((int)blockIdx.x >= cn || g >= count) return;
  copy_to_shared(&K, Kg);
  const int col = list ? list[g] : g;
  const float* m = model + (size_t)col * 13 * nz;
  const int nsamp = HE ? 2 * nz - 1 : nz;
  double* ts = sm_saha;                                        // the samples' temperatures
  SahaT* tt = reinterpret_cast<SahaT*>(sm_saha + nsamp);       // and their shared terms
  double* dzs = sm_saha + nsamp + nsamp * (sizeof(SahaT) / sizeof(double));   // HE: dz of step j
  double* t0s = dzs + nz;                                                     // and its start height
  if (HE) {
    const int top = nz - 1;
    for (int j = threadIdx.x; j < nz - 1; j += blockDim.x) {
      const int k = nz - 2 - j;
      dzs[j] = ((double)mget(m, nz, 12, k) - (double)mget(m, nz, 12, k + 1)) * 1000.0 * 100.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {   // the integration's own running height, added in its order
      double t0 = (double)mget(m, nz, 12, top) * 1000.0 * 100.0;
      for (int j = 0; j < nz - 1; ++j) {
        t0s[j] = t0;
        t0 = t0 + dzs[j];
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) ts[0] = (double)mget(m, nz, 0, top);
    for (int j = threadIdx.x; j < nz - 1; j += blockDim.x) {
      const int k = nz - 2 - j;
      const double tm0 = (double)mget(m, nz, 0, k + 1), tm1 = (double)mget(m, nz, 0, k);
      ts[2 * j + 1] = chain_tmid(t0s[j], dzs[j], tm0, tm1);
      ts[2 * j + 2] = tm1;
    }
  } else {
    for (int k = threadIdx.x; k < nz; k += blockDim.x) ts[k] = (double)mget(m, nz, 0, k);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nsamp; i += blockDim.x) tt[i] = saha_t(ts[i], K);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int e0 = K.lane_elem[lane], e1 = K.lane_elem[lane + 32], e2 = K.lane_elem[lane + 64];
  double2* out = sa + (size_t)blockIdx.x * nsamp * 96;
  const int wstride = (blockDim.x >> 5) * gridDim.y;
  for (int smp = (threadIdx.x >> 5) + blockIdx.y * (blockDim.x >> 5); smp < nsamp; smp += wstride) {
    const double T = ts[smp];
    const SahaT t = tt[smp];
    double2* o = out + (size_t)smp * 96;
    o[lane] = saha_elem<true>(e0, T, t, K, tb);
    o[lane + 32] = saha_elem<false>(e1, T, t, K, tb);
    o[lane + 64] = saha_elem<false>(e2, T, t, K, tb);
  }
}

// HE anchored at the height of least |log tau5| of the input model
// (RK4_INTEGRATION_LOG_LTAUM05 -> _MED, src/hydrostatic_tools.f90:226-346;
// FORWARD1D with HYDROSTATIC and HYDRO_TOP off, src/forward.f90:890-905):
// Pg kept there, RK4_LOG steps up to the top, then from the anchor down to
// the bottom with NELEC restarted from the anchor's Pe.  One warp per
// column (the synthesis-only entry points and SET_TAU use it; the
// inversion integrates from the top, k_chain).
__global__ void __launch_bounds__(128) k_chain_med(const Consts* __restrict__ Kg, const PFTable* __restrict__ tb,
                                                   int ncol, int nz, const float* model, float* mout,
                                                   double2* __restrict__ chem, int* __restrict__ status) {
  constexpr int L = 32;
  constexpr int NS = WarpSahaT<L>::NS;
  __shared__ Consts K;
  copy_to_shared(&K, Kg);
  __syncthreads();
  const int lane = threadIdx.x & (L - 1);
  const int col = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) / L);
  if (col >= ncol) return;
  const float* m = model + (size_t)col * 13 * nz;
  float* mo = mout + (size_t)col * 13 * nz;
  double2* ch = chem + (size_t)col * nz;
  // the anchor from the input model, before mo (which may alias m) changes
  int iz = 0;
  for (int k = 1; k < nz; ++k)
    if (fabsf(mget(m, nz, 11, k)) < fabsf(mget(m, nz, 11, iz))) iz = k;
  __syncwarp();
  if (mo != m)
    for (int i = lane; i < 13 * nz; i += L) mo[i] = m[i];
  __syncwarp();
  double ab[NS];
#pragma unroll
  for (int j = 0; j < NS; ++j) ab[j] = K.lane_elem[L * j + lane] >= 0 ? K.ab10[K.lane_elem[L * j + lane]] : 0.0;
  int st = 0;
  const double tz = (double)mget(mo, nz, 0, iz);
  double nelec = (double)mget(mo, nz, 3, iz) / KBOL / tz;
  const double ua = log((double)mget(mo, nz, 1, iz));
  WarpSahaT<L> w;
  saha_prepare(w, tz, K, tb, lane);
  double nelec_down;
  {
    const RhoOut r = get_rho_warp(w, ab, exp(ua), nelec, K, lane);
    st |= r.status;
    nelec_down = r.pelec / KBOL / tz;
    __syncwarp();
    if (lane == 0) {
      const float pel = (float)r.pelec;
      mo[1 * nz + iz] = (float)exp(ua);
      mo[2 * nz + iz] = (float)r.dens;
      mo[3 * nz + iz] = pel;
      mo[4 * nz + iz] = (float)r.molecw;
      ch[iz] = make_double2(r.nhyd, (double)pel / KBOL / tz);
    }
  }
  // the Saha buffer holds T(kf) when a step from kf to kt starts
  auto step = [&](int kf, int kt, double& t0, double& u0) {
    const double dz = ((double)mget(m, nz, 12, kt) - (double)mget(m, nz, 12, kf)) * 1000.0 * 100.0;
    const double tm0 = (double)mget(m, nz, 0, kf), tm1 = (double)mget(m, nz, 0, kt);
    const double it1 = t0 + dz / 2.0;
    const double tmid = tm0 / dz * (t0 + dz - it1) + tm1 / dz * (it1 - t0);
    double kk[4] = {0.0, 0.0, 0.0, 0.0};
    double u1 = 0.0;
#pragma unroll 1
    for (int stg = 0; stg < 5; ++stg) {
      if (stg == 1 || stg == 3) saha_prepare(w, stg == 1 ? tmid : tm1, K, tb, lane);
      const double tem = stg == 0 ? tm0 : (stg < 3 ? tmid : tm1);
      const double y = stg == 0 ? u0 : (stg == 1 ? u0 + kk[0] / 2.0 : (stg == 2 ? u0 + kk[1] / 2.0 : (stg == 3 ? u0 + kk[2] : u1)));
      const RhoOut q = get_rho_warp(w, ab, exp(y), nelec, K, lane);
      st |= q.status;
      if (stg < 4) {
        const double d = (-q.molecw * MAMU * GRAV / (KBOL * tem)) * dz;
        kk[stg] = d;
        if (stg == 3) u1 = u0 + 1.0 / 6.0 * (kk[0] + 2.0 * kk[1] + 2.0 * kk[2] + kk[3]);
      } else if (lane == 0) {
        const float pel = (float)q.pelec;
        mo[1 * nz + kt] = (float)exp(u1);
        mo[2 * nz + kt] = (float)q.dens;
        mo[3 * nz + kt] = pel;
        mo[4 * nz + kt] = (float)q.molecw;
        ch[kt] = make_double2(q.nhyd, (double)pel / KBOL / tm1);
      }
    }
    u0 = u1;
    t0 = t0 + dz;
  };
  double t0 = (double)mget(m, nz, 12, iz) * 1000.0 * 100.0, u0 = ua;
  for (int k = iz + 1; k < nz; ++k) step(k - 1, k, t0, u0);
  if (iz > 0) {
    t0 = (double)mget(m, nz, 12, iz) * 1000.0 * 100.0;
    u0 = ua;
    nelec = nelec_down;
    saha_prepare(w, tz, K, tb, lane);
    for (int k = iz - 1; k >= 0; --k) step(k + 1, k, t0, u0);
  }
  if (lane == 0 && status) status[col] = st;
}

// ------------------------------------------------------------------ k_opac
// One thread per (column, height): every per-height quantity of the slab.
// KC5 and the boundary flag (src/forward.f90:926-931), KC of each region at
// its main line (:940), KLIN and the damping of every line (:949-951), the
// Doppler width, velocity shift and field geometry of GET_ABS_MAT
// (src/absorption_matrix.f90:914-991, :1018).
__global__ void __launch_bounds__(256) k_opac(const DevParams* __restrict__ Pg, const Consts* __restrict__ Kg,
                                              int ncol, const float* __restrict__ mout,
                                              const double2* __restrict__ chem, float* __restrict__ slab,
                                              const int* __restrict__ list = nullptr,
                                              const int* __restrict__ nlist = nullptr) {
  __shared__ DevParams P;
  __shared__ Consts K;
  const size_t total = (size_t)(list ? *nlist : ncol) * Pg->nz;
  if ((size_t)blockIdx.x * blockDim.x >= total) return;
  copy_to_shared(&P, Pg);
  copy_to_shared(&K, Kg);
  __syncthreads();
  const int nz = P.nz, sw = P.sw;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int idx = (int)(t / nz), k = (int)(t % nz);
    const int col = list ? list[idx] : idx;
    const size_t i = (size_t)col * nz + k;
    const float* m = mout + (size_t)col * 13 * nz;
    const double2 c = chem[i];
    const double nhyd = c.x, nelec = c.y;
    const float Tf = mget(m, nz, 0, k);
    const double T = (double)Tf;
    const double dz = (k == nz - 1) ? 1e5 * fabs((double)mget(m, nz, 12, k) - (double)mget(m, nz, 12, k - 1))
                                    : 1e5 * fabs((double)mget(m, nz, 12, k + 1) - (double)mget(m, nz, 12, k));
    float* row = slab + i * sw;
    const double kc5 = opac_continuum(T, nelec, nhyd, P.cont[P.nreg]) / nhyd * (1.0 / MAMU);
    row[0] = Tf;
    row[1] = (kc5 < KC5THRESHOLD) ? 0.0f : 1.0f;
    row[2] = (float)kc5;
    row[3] = mget(m, nz, 2, k);
    for (int r = 0; r < P.nreg; ++r) row[4 + r] = (float)(opac_continuum(T, nelec, nhyd, P.cont[r]) * dz);
    // field geometry, src/absorption_matrix.f90:919-991
    {
      const double x = mget(m, nz, 5, k), y = mget(m, nz, 6, k), z = mget(m, nz, 7, k);
      const double x2 = x * x, y2 = y * y, z2 = z * z;
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
    const double vz = (double)mget(m, nz, 10, k);
    for (int b = 0; b < P.nlu; ++b) {
      const LineP& L = P.lu[b];
      const double klin = opac_line(L, T, nelec, nhyd, K);
      const double damp = get_damping(L, nhyd, T);
      const double dldop = 1e3 * (sqrt(L.vdk * T) * L.l0 / LIGHT);
      const double dlv = -1e3 * L.l0 * vz / LIGHT;
      float* q = row + slab_line(P.nreg) + 4 * b;
      q[0] = (float)(klin * dz);
      q[1] = (float)damp;
      q[2] = (float)(1.0 / dldop);
      q[3] = (float)(dlv - L.wdif);
    }
  }
}

// ----------------------------------------------------------------- k_synth
// One height of OLD_ANALYTICAL_SOLVER (src/rtesolver.f90:163-187): I_k =
// (1 - O) S e0 + O I_{k-1}, om0 = 1 - O(1,1).
__device__ __forceinline__ void rte_step(const float O[16], float om0, float S, float& I0, float& I1, float& I2,
                                         float& I3) {
  const float n0 = fmaf(om0, S, fmaf(O[0], I0, fmaf(O[1], I1, fmaf(O[2], I2, O[3] * I3))));
  const float n1 = fmaf(-O[4], S, fmaf(O[4], I0, fmaf(O[5], I1, fmaf(O[6], I2, O[7] * I3))));
  const float n2 = fmaf(-O[8], S, fmaf(O[8], I0, fmaf(O[9], I1, fmaf(O[10], I2, O[11] * I3))));
  const float n3 = fmaf(-O[12], S, fmaf(O[12], I0, fmaf(O[13], I1, fmaf(O[14], I2, O[15] * I3))));
  I0 = n0;
  I1 = n1;
  I2 = n2;
  I3 = n3;
}

// The synthesis of column col from its slab staged in shared memory (sm),
// one thread per wavelength l.
__device__ __forceinline__ void synth_column(const DevParams& P, const LamP* __restrict__ lam,
                                             const float* __restrict__ gain, const float* sm, int col,
                                             double* __restrict__ syn, float* mout, int* __restrict__ status) {
  const int nz = P.nz, sw = P.sw;
  const int l = threadIdx.x;
  if (l >= P.numw) return;
  if (l == 0) {
    // log tau5 from the top, src/forward.f90:1000-1006 (REAL*4 accumulation)
    float* mo = mout + (size_t)col * 13 * nz;
    float tau = 1e-9f;
    mo[11 * nz + nz - 1] = log10f(tau);
    for (int k = nz - 2; k >= 0; --k) {
      const float a = (sm[k * sw + 2] * sm[k * sw + 3] + sm[(k + 1) * sw + 2] * sm[(k + 1) * sw + 3]) / 2.0f;
      const double b = ((double)mo[12 * nz + k + 1] - (double)mo[12 * nz + k]) * 1000.0 * 100.0;
      tau = (float)((double)tau + (double)a * b);
      mo[11 * nz + k] = log10f(tau);
    }
  }
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
    float tI = row[4 + r], tQ = 0.f, tU = 0.f, tV = 0.f, rQ = 0.f, rU = 0.f, rV = 0.f;
    for (int b = 0; b < nb; ++b) {
      const float* q = row + loff + 4 * (lb + b);
      const float kldz = q[0], a = q[1], idd = q[2];
      const float x0 = lp.wave + q[3];
      float h0 = 0.f, h1 = 0.f, h2 = 0.f, f0 = 0.f, f1 = 0.f, f2 = 0.f;
      // components are stored sigma_red (dM=-1), pi, sigma_blue (dM=+1)
      int c = P.lu_c0[lb + b];
      const int e0 = c + P.lu_nt[lb + b][0], e1 = e0 + P.lu_nt[lb + b][1], e2 = e1 + P.lu_nt[lb + b][2];
      for (; c < e0; ++c) {
        float h, f;
        voigt_f32(a, fmaf(P.comp_shift[c], B, x0) * idd, h, f);
        h0 = fmaf(P.comp_str[c], h, h0);
        f0 = fmaf(P.comp_str[c], f, f0);
      }
      for (; c < e1; ++c) {
        float h, f;
        voigt_f32(a, fmaf(P.comp_shift[c], B, x0) * idd, h, f);
        h1 = fmaf(P.comp_str[c], h, h1);
        f1 = fmaf(P.comp_str[c], f, f1);
      }
      for (; c < e2; ++c) {
        float h, f;
        voigt_f32(a, fmaf(P.comp_shift[c], B, x0) * idd, h, f);
        h2 = fmaf(P.comp_str[c], h, h2);
        f2 = fmaf(P.comp_str[c], f, f2);
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
    float O[16], om0 = 0.0f;
    if (!(isfinite(tI) && isfinite(tQ) && isfinite(tU) && isfinite(tV) && isfinite(rQ) && isfinite(rU) &&
          isfinite(rV))) {
      bad = 1;   // the reference replaces a non-finite matrix by the identity
#pragma unroll
      for (int i = 0; i < 16; ++i) O[i] = (i % 5 == 0) ? 1.f : 0.f;
    } else {
      evol_f32(tI, tQ, tU, tV, rQ, rU, rV, O, om0);
    }
    rte_step(O, om0, S, I0, I1, I2, I3);
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

// One CTA per column, one thread per wavelength, FP32: the Stokes synthesis
// of the column's slab.  With a list, the CTAs walk list[0, *nlist) (the
// occupied slots of an inversion pool) with a grid stride.
__global__ void __launch_bounds__(MAXNUMW) k_synth(const DevParams* __restrict__ Pg, const LamP* __restrict__ lam,
                                                   const float* __restrict__ gain, int ncol,
                                                   const float* __restrict__ slab, double* __restrict__ syn,
                                                   float* mout, int* __restrict__ status,
                                                   const int* __restrict__ list = nullptr,
                                                   const int* __restrict__ nlist = nullptr) {
  extern __shared__ float4 sm_synth4[];
  __shared__ DevParams P;
  const int count = list ? *nlist : ncol;
  if ((int)blockIdx.x >= count) return;
  copy_to_shared(&P, Pg);
  const int nz = Pg->nz, sw = Pg->sw;
  for (int idx = blockIdx.x; idx < count; idx += gridDim.x) {
    const int col = list ? list[idx] : idx;
    __syncthreads();   // P in place; the previous column's slab no longer read
    // stage the column's slab (nz*sw floats, 16-byte rows) in shared memory
    const float4* src = reinterpret_cast<const float4*>(slab + (size_t)col * nz * sw);
    const int n4 = nz * sw / 4;
    for (int i = threadIdx.x; i < n4; i += blockDim.x) sm_synth4[i] = __ldg(src + i);
    __syncthreads();
    synth_column(P, lam, gain, reinterpret_cast<const float*>(sm_synth4), col, syn, mout, status);
  }
}

// ------------------------------------------------------ response functions
// RF slab row = the synthesis row followed by the derivative inputs:
//   dkc_t*dz, dkc_p*dz per region; per used line dkl_t*dz, dkl_p*dz,
//   ddam_t, ddam_p; per field component i (x, y, z) the derivatives of the
//   five geometry factors (0.25 cgf, 0.5 sgf, sgf c2p, sgf s2p, 0.5 cosg);
//   dB/dB_i (3); hydrostatic factor c_K (below) and Pg_K.
__host__ __device__ inline int rf_base(int nreg, int nlu) { return 4 + nreg + 6 + 4 * nlu; }
__host__ __device__ inline int rf_dkc(int nreg, int nlu) { return rf_base(nreg, nlu); }
__host__ __device__ inline int rf_dline(int nreg, int nlu) { return rf_base(nreg, nlu) + 2 * nreg; }
__host__ __device__ inline int rf_dgeo(int nreg, int nlu) { return rf_dline(nreg, nlu) + 4 * nlu; }
__host__ __device__ inline int rf_db(int nreg, int nlu) { return rf_dgeo(nreg, nlu) + 15; }
__host__ __device__ inline int rf_he(int nreg, int nlu) { return rf_db(nreg, nlu) + 3; }
__host__ __device__ inline int rf_w(int nreg, int nlu) { return (rf_he(nreg, nlu) + 2 + 3) & ~3; }

// Node layout of the Jacobian: parameter slots T|Pg, Pg|T, Bx, By, Bz, v_z
// (reference parameters 1, 2, 4, 5, 6, 7); slot p owns nodes [n0[p], n0[p]+nj[p]).
constexpr int NSLOT = 6;
constexpr int MAXNP = 64;
struct RFConf {
  int np;
  int nj[NSLOT], n0[NSLOT];
};

// One warp per (column, height), FP64, lanes over the elements: the
// chemistry derivatives of GET_DNHYDDTEMP at the (T, Pg, NELEC) that
// FORWARD1D passes to it (src/forward.f90:917-918).
__global__ void __launch_bounds__(128) k_chemder(const DevParams* __restrict__ Pg, const Consts* __restrict__ Kg,
                                                 const PFTable* __restrict__ tb, const PFDTable* __restrict__ td,
                                                 int ncol, const float* __restrict__ mout,
                                                 const double2* __restrict__ chem, double4* __restrict__ chemd,
                                                 const int* __restrict__ list, const int* __restrict__ nlist) {
  __shared__ Consts K;
  copy_to_shared(&K, Kg);
  __syncthreads();
  const int nz = Pg->nz;
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const size_t total = (size_t)(list ? *nlist : ncol) * nz;
  for (size_t j = (size_t)blockIdx.x * wpb + (threadIdx.x >> 5); j < total; j += (size_t)gridDim.x * wpb) {
    const int k = (int)(j % nz), col = list ? list[j / nz] : (int)(j / nz);
    const size_t i = (size_t)col * nz + k;
    const float* m = mout + (size_t)col * 13 * nz;
    const ChemDer cd = chem_der_warp((double)mget(m, nz, 0, k), (double)mget(m, nz, 1, k), chem[i].y, K, tb, td, lane);
    if (lane == 0) chemd[i] = make_double4(cd.dne_p, cd.dnh_p, cd.dne_t, cd.dnh_t);
  }
}

// One thread per (column, height), FP64: the synthesis slab row of k_opac
// plus the derivative inputs of the response functions.  The hydrostatic
// factor of GET_HYD_DERIVATIVES (:1050-1057) is stored as
// c_K = DPGDTK_HE(I) / Pg(I) = -(Pg_K mu_K)_REAL*4 CTE / T_K^2 / Pg_K.
__global__ void __launch_bounds__(256) k_opac_rf(const DevParams* __restrict__ Pg, const Consts* __restrict__ Kg,
                                                 int ncol, const float* __restrict__ mout,
                                                 const double2* __restrict__ chem, const double4* __restrict__ chemd,
                                                 float* __restrict__ slab, const int* __restrict__ list,
                                                 const int* __restrict__ nlist) {
  __shared__ DevParams P;
  __shared__ Consts K;
  copy_to_shared(&P, Pg);
  copy_to_shared(&K, Kg);
  __syncthreads();
  const int nz = P.nz, nreg = P.nreg, nlu = P.nlu;
  const int sw = rf_w(nreg, nlu);
  const size_t total = (size_t)(list ? *nlist : ncol) * nz;
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(j % nz), col = list ? list[j / nz] : (int)(j / nz);
    const size_t i = (size_t)col * nz + k;
    const float* m = mout + (size_t)col * 13 * nz;
    const double2 c = chem[i];
    const double nhyd = c.x, nelec = c.y;
    const double4 d4 = chemd[i];
    ChemDer cd;
    cd.dne_p = d4.x;
    cd.dnh_p = d4.y;
    cd.dne_t = d4.z;
    cd.dnh_t = d4.w;
    const float Tf = mget(m, nz, 0, k);
    const double T = (double)Tf;
    const double dz = (k == nz - 1) ? 1e5 * fabs((double)mget(m, nz, 12, k) - (double)mget(m, nz, 12, k - 1))
                                    : 1e5 * fabs((double)mget(m, nz, 12, k + 1) - (double)mget(m, nz, 12, k));
    float* row = slab + i * sw;
    {
      const double kc5 = opac_continuum(T, nelec, nhyd, P.cont[P.nreg]) / nhyd * (1.0 / MAMU);
      row[0] = Tf;
      row[1] = (kc5 < KC5THRESHOLD) ? 0.0f : 1.0f;
      row[2] = (float)kc5;
      row[3] = mget(m, nz, 2, k);
      const double x = mget(m, nz, 5, k), y = mget(m, nz, 6, k), z = mget(m, nz, 7, k);
      const double x2 = x * x, y2 = y * y, z2 = z * z;
      const double b2 = x2 + y2 + z2, b = sqrt(b2);
      const double xm = x2 - y2, xp = x2 + y2;
      double cosg = 0, cgf = 1, sgf = 1, c2p = 0, s2p = 0;
      double dcgf[3] = {0, 0, 0}, dc2p[3] = {0, 0, 0}, ds2p[3] = {0, 0, 0}, dcg[3] = {0, 0, 0}, db[3] = {0, 0, 0};
      if (b > 0) {
        cosg = z / b;
        cgf = 1 + z2 / b2;
        sgf = 1 - z2 / b2;
        // src/absorption_matrix.f90:1852-1873 (0/0 for Bx = By = 0 < B, as there)
        dcgf[0] = -2.0 * x * z2 / b2 / b2;
        dcgf[1] = -2.0 * y * z2 / b2 / b2;
        dcgf[2] = (2.0 * z * (b2 - z2)) / b2 / b2;
        dc2p[0] = 4.0 * x * y2 / xp / xp;
        dc2p[1] = -4.0 * y * x2 / xp / xp;
        ds2p[0] = -2.0 * y * xm / xp / xp;
        ds2p[1] = 2.0 * x * xm / xp / xp;
        dcg[0] = -(z * x) / b / b2;
        dcg[1] = -(z * y) / b / b2;
        dcg[2] = (1.0 - cosg * cosg) / b;
        db[0] = x / b;
        db[1] = y / b;
        db[2] = z / b;
      }
      if (x != 0 || y != 0) {
        c2p = xm / xp;
        s2p = 2. * x * y / xp;
      }
      float* g = row + slab_geo(nreg);
      g[0] = (float)(0.25 * cgf);
      g[1] = (float)(0.5 * sgf);
      g[2] = (float)(sgf * c2p);
      g[3] = (float)(sgf * s2p);
      g[4] = (float)(0.5 * cosg);
      g[5] = (float)b;
      float* dg = row + rf_dgeo(nreg, nlu);
      for (int q = 0; q < 3; ++q) {
        const double dsgf = -dcgf[q];
        dg[5 * q + 0] = (float)(0.25 * dcgf[q]);
        dg[5 * q + 1] = (float)(0.5 * dsgf);
        dg[5 * q + 2] = (float)(dsgf * c2p + sgf * dc2p[q]);
        dg[5 * q + 3] = (float)(dsgf * s2p + sgf * ds2p[q]);
        dg[5 * q + 4] = (float)(0.5 * dcg[q]);
        row[rf_db(nreg, nlu) + q] = (float)db[q];
      }
      double ck = 0.0;
      const float pgk = mget(m, nz, 1, k);
      if (k > 0) {
        const double cte =
            MAMU / KBOL * GRAV * ((double)mget(m, nz, 12, k) - (double)mget(m, nz, 12, k - 1)) * 1.0e3 * 1.0e2;
        const float pm = pgk * mget(m, nz, 4, k);
        ck = -((double)pm * cte / T / T) / (double)pgk;
      }
      row[rf_he(nreg, nlu)] = (float)ck;
      row[rf_he(nreg, nlu) + 1] = pgk;
    }
    for (int r = 0; r < nreg; ++r) {
      row[4 + r] = (float)(opac_continuum(T, nelec, nhyd, P.cont[r]) * dz);
      double dt, dp;
      cont_der(T, nelec, nhyd, P.cont[r], cd, dt, dp);
      row[rf_dkc(nreg, nlu) + 2 * r] = (float)(dt * dz);
      row[rf_dkc(nreg, nlu) + 2 * r + 1] = (float)(dp * dz);
    }
    for (int b = 0; b < nlu; ++b) {
      const LineP& L = P.lu[b];
      const double klin = opac_line(L, T, nelec, nhyd, K);
      const double damp = get_damping(L, nhyd, T);
      const double dldop = 1e3 * (sqrt(L.vdk * T) * L.l0 / LIGHT);
      const double dlv = -1e3 * L.l0 * (double)mget(m, nz, 10, k) / LIGHT;
      float* q = row + slab_line(nreg) + 4 * b;
      q[0] = (float)(klin * dz);
      q[1] = (float)damp;
      q[2] = (float)(1.0 / dldop);
      q[3] = (float)(dlv - L.wdif);
      double dkt, dkp, ddt, ddp;
      line_der(L, T, nelec, nhyd, cd, K, dkt, dkp);
      damp_der(L, nhyd, T, cd, ddt, ddp);
      float* d = row + rf_dline(nreg, nlu) + 4 * b;
      d[0] = (float)(dkt * dz);
      d[1] = (float)(dkp * dz);
      d[2] = (float)ddt;
      d[3] = (float)ddp;
    }
  }
}

// Offset (floats, 16-byte aligned) of the per-thread sums of k_synth_rf
// behind the slab (nz x sw), the coefficient table (nz x np) and the node
// accumulators (np x 4 x nthr); the block's dynamic shared memory is that
// offset plus six float4 a thread.
__host__ __device__ __forceinline__ int rf_sums_off(int nz, int sw, int np, int nthr) {
  return (nz * sw + nz * np + np * 4 * nthr + 3) & ~3;
}

// A thread's own float4 in shared memory, stored and loaded as volatile
// instructions: the loads are issued where they stand, so the values are not
// kept in registers between the store and the loads.
__device__ __forceinline__ void sts4(float4* p, float a, float b, float c, float d) {
  asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(p))),
               "f"(a), "f"(b), "f"(c), "f"(d));
}
__device__ __forceinline__ float4 lds4(const float4* p) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(static_cast<unsigned>(__cvta_generic_to_shared(p))));
  return v;
}

// Linear maps from the per-type (sigma_red, pi, sigma_blue) sums of one line
// to the seven matrix elements (eta_I,Q,U,V, rho_Q,U,V), the grouping of the
// component accumulation of src/absorption_matrix.f90:1948-2278.
struct Geo {
  float g1, g2, g3, g4, g5;
};
__device__ __forceinline__ void lmap(const Geo& g, const float h[3], const float f[3], float o[7]) {
  const float hs = h[0] + h[2], fs = f[0] + f[2];
  const float hl = 0.5f * h[1] - 0.25f * hs, fl = 0.5f * f[1] - 0.25f * fs;
  o[0] = g.g1 * hs + g.g2 * h[1];
  o[1] = g.g3 * hl;
  o[2] = g.g4 * hl;
  o[3] = g.g5 * (h[0] - h[2]);
  o[4] = g.g3 * fl;
  o[5] = g.g4 * fl;
  o[6] = g.g5 * (f[0] - f[2]);
}

// One CTA per column, one thread per wavelength, FP32: the synthesis of
// k_synth plus, per height, the derivatives of the seven optical depths for
// the six parameters (WDEV, src/absorption_matrix.f90:1717-2642), the local
// response functions of OLD_ANALYTICAL_SOLVER (src/rtesolver.f90:194-260)
// and their forward accumulation into the node Jacobian:
//   D_j <- O_K D_j + coef(K, j) RF_p(K)
// which equals OLD_DSYN_PROPAGATION (src/forward.f90:511-548) followed by
// the hat-function contraction of CALCULATE_EQUIVALENT_DSYN (:552-681).
// Hydrostatic mode adds the global T term of :218-232 through the
// recurrence H_K = O_K H_{K-1} + RF_Pg(K) Pg_K (skipped where O_K(1,1) <=
// 1e-5), RF_T(K) += c_K O_K H_{K-1}, and evaluates the B and v_z terms with
// the layer's outgoing Stokes vector, as the reference does (STKIN is
// reassigned at :230).  Layers that take the boundary condition have no
// response and reset the accumulators (their operator is taken as 0).
// Shared memory: the slab, the coefficient table (nz x np) and the node
// accumulators (np x 4 x blockDim).
//
// FULL: the response functions at every height instead of the node
// Jacobian (NJ = NZ for every parameter): the local RFs of each layer go to
// jac in the (NFREQ, 6 NZ) layout and the layer's operator to oscr
// ((nz, 16, NUMW) per column, zero where the boundary condition is taken);
// k_rf_prop then applies the products of the operators above each layer.
// MAXT: the block-size bound, 256 (two blocks per SM) up to 256
// wavelengths, 512 (one) up to 512; both hold 128 registers a thread.
// BLEND: regions with blended lines are present and every region runs the
// general path below; without, only the single-line path is compiled in,
// which keeps the general path's register demand out of the kernel.
template <bool HE, bool FULL, int MAXT, bool BLEND>
__global__ void __launch_bounds__(MAXT, (MAXT <= 256 ? 2 : 1)) k_synth_rf(const DevParams* __restrict__ Pg, const RFConf* __restrict__ Rg,
                                                  const LamP* __restrict__ lam, const float* __restrict__ gain,
                                                  int ncol, const float* __restrict__ slab,
                                                  const float* __restrict__ coefg, double* __restrict__ syn,
                                                  float* __restrict__ jac, float* __restrict__ oscr, float* mout,
                                                  int* __restrict__ status, const int* __restrict__ list,
                                                  const int* __restrict__ nlist) {
  if (list && (int)blockIdx.x >= *nlist) return;
  extern __shared__ float4 sm_rf4[];
  __shared__ DevParams P;
  __shared__ RFConf C;
  __shared__ unsigned inf_mask[2];
  copy_to_shared(&P, Pg);
  if (!FULL) copy_to_shared(&C, Rg);
  const int col = list ? list[blockIdx.x] : (int)blockIdx.x;
  const int nz = Pg->nz, nreg = Pg->nreg, nlu = Pg->nlu, np = FULL ? 0 : Rg->np;
  const int sw = rf_w(nreg, nlu);
  const int nthr = blockDim.x;
  float* sm = reinterpret_cast<float*>(sm_rf4);
  float* coef = sm + nz * sw;
  float* Dacc = coef + nz * np;
  // the per-wavelength sums of the single-line path, six float4 a thread
  // (vector v of thread l at sums[v * nthr + l]), after the accumulators
  float4* sums = reinterpret_cast<float4*>(sm + rf_sums_off(nz, sw, np, nthr));
  {
    const float4* src = reinterpret_cast<const float4*>(slab + (size_t)col * nz * sw);
    const int n4 = nz * sw / 4;
    for (int i = threadIdx.x; i < n4; i += nthr) sm_rf4[i] = __ldg(src + i);
    if (!FULL) {
      for (int i = threadIdx.x; i < nz * np; i += nthr) coef[i] = __ldg(coefg + i);
      for (int i = threadIdx.x; i < np * 4 * nthr; i += nthr) Dacc[i] = 0.0f;
    }
    if (threadIdx.x < 2) inf_mask[threadIdx.x] = 0u;
  }
  const size_t fstride = (size_t)4 * Pg->numw;   // NFREQ
  float* jcol = jac + (size_t)col * (FULL ? NSLOT * nz : 0) * fstride;
  float* ocol = FULL ? oscr + (size_t)col * nz * 16 * Pg->numw : nullptr;
  __syncthreads();
  const int l = threadIdx.x;
  const bool active = l < P.numw;
  if (l == 0) {
    // log tau5, src/forward.f90:1000-1006 (as k_synth)
    float* mo = mout + (size_t)col * 13 * nz;
    float tau = 1e-9f;
    mo[11 * nz + nz - 1] = log10f(tau);
    for (int k = nz - 2; k >= 0; --k) {
      const float a = (sm[k * sw + 2] * sm[k * sw + 3] + sm[(k + 1) * sw + 2] * sm[(k + 1) * sw + 3]) / 2.0f;
      const double b = ((double)mo[12 * nz + k + 1] - (double)mo[12 * nz + k]) * 1000.0 * 100.0;
      tau = (float)((double)tau + (double)a * b);
      mo[11 * nz + k] = log10f(tau);
    }
  }
  const LamP lp = lam[active ? l : 0];
  const int r = lp.reg;
  const int nb = P.reg_nb[r], lb = P.reg_lb[r];
  const int goff = slab_geo(nreg), loff = slab_line(nreg);
  const int dkoff = rf_dkc(nreg, nlu) + 2 * r, dloff = rf_dline(nreg, nlu), dgoff = rf_dgeo(nreg, nlu);
  const int dboff = rf_db(nreg, nlu), heoff = rf_he(nreg, nlu);
  float I0 = 0.f, I1 = 0.f, I2 = 0.f, I3 = 0.f;
  float H[4] = {0.f, 0.f, 0.f, 0.f};
  int bad = 0;
  for (int k = 0; active && k < nz; ++k) {
    const float* row = sm + k * sw;
    const float T = row[0];
    const float q = lp.c2 / T;
    const float em1 = expm1f(q);
    const float S = lp.c1 / em1;
    if (k == 0 || row[1] != 0.0f) {   // SET_BOUNDARY
      I0 = S;
      I1 = I2 = I3 = 0.f;
      if (FULL) {
        const int nw = P.numw;
#pragma unroll
        for (int p = 0; p < NSLOT; ++p)
#pragma unroll
          for (int c = 0; c < 4; ++c) jcol[((size_t)p * nz + k) * fstride + c * nw + l] = 0.0f;
#pragma unroll
        for (int i = 0; i < 16; ++i) ocol[((size_t)k * 16 + i) * nw + l] = 0.0f;
      } else {
        for (int j = 0; j < np; ++j)
#pragma unroll
          for (int c = 0; c < 4; ++c) Dacc[(j * 4 + c) * nthr + l] = 0.0f;
      }
      continue;
    }
    const Geo g{row[goff], row[goff + 1], row[goff + 2], row[goff + 3], row[goff + 4]};
    const float B = row[goff + 5];
    const float halfT = 0.5f / T;
    if (!BLEND) {
      // One line in every region (no blends): each parameter's optical-depth
      // derivatives are formed from the line's per-type sums when its
      // response is taken, in a runtime loop over the parameters -- one
      // copy of the directional derivative and of the node update, and no
      // 6 x 7 array held across the operator algebra.  The arithmetic is
      // that of the general path below, expression for expression.
      const float* qq = row + loff + 4 * lb;
      const float kldz = qq[0], a = qq[1], idd = qq[2];
      const float x0 = lp.wave + qq[3];
      float hh[3] = {0, 0, 0}, ff[3] = {0, 0, 0}, av[3] = {0, 0, 0}, ca[3] = {0, 0, 0};
      float avu[3] = {0, 0, 0}, cau[3] = {0, 0, 0}, avs[3] = {0, 0, 0}, cas[3] = {0, 0, 0};
      {
        int c = P.lu_c0[lb];
#pragma unroll
        for (int t = 0; t < 3; ++t) {
          const int e = c + P.lu_nt[lb][t];
          for (; c < e; ++c) {
            const float shf = P.comp_shift[c], st = P.comp_str[c];
            const float u = fmaf(shf, B, x0) * idd;
            float h, f;
            voigt_f32(a, u, h, f);
            const float dhv = 2.0f * fmaf(a, f, -u * h);
            const float dha = 2.0f * (fmaf(a, h, u * f) - 0.56418958354775628f);
            hh[t] = fmaf(st, h, hh[t]);
            ff[t] = fmaf(st, f, ff[t]);
            const float sv = st * dhv, sa = st * dha;
            av[t] += sv;
            ca[t] += sa;
            avu[t] = fmaf(sv, u, avu[t]);
            cau[t] = fmaf(sa, u, cau[t]);
            avs[t] = fmaf(sv, shf, avs[t]);
            cas[t] = fmaf(sa, shf, cas[t]);
          }
        }
      }
      // the sums wait in shared memory through the operator algebra and are
      // read back per parameter: 24 registers fewer across the loop below
      float4* su = sums + l;
      sts4(su, hh[0], hh[1], hh[2], ff[0]);
      sts4(su + nthr, ff[1], ff[2], av[0], av[1]);
      sts4(su + 2 * nthr, av[2], ca[0], ca[1], ca[2]);
      sts4(su + 3 * nthr, avu[0], avu[1], avu[2], cau[0]);
      sts4(su + 4 * nthr, cau[1], cau[2], avs[0], avs[1]);
      sts4(su + 5 * nthr, avs[2], cas[0], cas[1], cas[2]);
      float tI = row[4 + r], tQ, tU, tV, rQ, rU, rV;
      {
        const float hs = hh[0] + hh[2], fs = ff[0] + ff[2];
        const float hl = 0.5f * hh[1] - 0.25f * hs, fl = 0.5f * ff[1] - 0.25f * fs;
        tI = fmaf(kldz, g.g1 * hs + g.g2 * hh[1], tI);
        tQ = fmaf(kldz, g.g3 * hl, 0.f);
        tU = fmaf(kldz, g.g4 * hl, 0.f);
        tV = fmaf(kldz, g.g5 * (hh[0] - hh[2]), 0.f);
        rQ = fmaf(kldz, g.g3 * fl, 0.f);
        rU = fmaf(kldz, g.g4 * fl, 0.f);
        rV = fmaf(kldz, g.g5 * (ff[0] - ff[2]), 0.f);
      }
      const float* dl = row + dloff + 4 * lb;
      const float dkt = dl[0], dkp = dl[1], ddt = dl[2], ddp = dl[3];
      float O[16], om0 = 0.0f;
      EvolSt es;
      const bool fin = isfinite(tI) && isfinite(tQ) && isfinite(tU) && isfinite(tV) && isfinite(rQ) &&
                       isfinite(rU) && isfinite(rV);
      if (!fin) {
        bad = 1;
#pragma unroll
        for (int i = 0; i < 16; ++i) O[i] = (i % 5 == 0) ? 1.f : 0.f;
      } else {
        evol_state(tI, tQ, tU, tV, rQ, rU, rV, O, om0, es);
      }
      const float n0 = fmaf(om0, S, fmaf(O[0], I0, fmaf(O[1], I1, fmaf(O[2], I2, O[3] * I3))));
      const float n1 = fmaf(-O[4], S, fmaf(O[4], I0, fmaf(O[5], I1, fmaf(O[6], I2, O[7] * I3))));
      const float n2 = fmaf(-O[8], S, fmaf(O[8], I0, fmaf(O[9], I1, fmaf(O[10], I2, O[11] * I3))));
      const float n3 = fmaf(-O[12], S, fmaf(O[12], I0, fmaf(O[13], I1, fmaf(O[14], I2, O[15] * I3))));
      // the operator products with the incoming vector (T, Pg; every
      // parameter without HE) -- with HE the B and v_z responses use the
      // outgoing one, switched to at p = 2
      EvolW v;
      if (fin) {
        const float win[4] = {I0 - S, I1, I2, I3};
        evol_w(es, O, win, v);
      }
      const float dS = lp.c1 * (q / T) * ((em1 + 1.0f) / (em1 * em1));
      float OH[4] = {0.f, 0.f, 0.f, 0.f}, ck = 0.f, pgk = 0.f;
      bool prop = false;
      if (HE) {
        ck = row[heoff];
        pgk = row[heoff + 1];
        prop = O[0] > 1.0e-5f;
#pragma unroll
        for (int i = 0; i < 4; ++i)
          OH[i] = prop ? O[4 * i] * H[0] + O[4 * i + 1] * H[1] + O[4 * i + 2] * H[2] + O[4 * i + 3] * H[3] : H[i];
      }
      const float* ckr = FULL ? nullptr : coef + k * np;
#pragma unroll 1
      for (int p = 0; p < NSLOT; ++p) {
        // every parameter's optical-depth derivatives in one form:
        //   dt = A lmap(GA, hh, ff) + B lmap(g, U, V), dt[0] += C0
        const float4 s0 = lds4(su), s1 = lds4(su + nthr), s2 = lds4(su + 2 * nthr);
        const float hh[3] = {s0.x, s0.y, s0.z}, ff[3] = {s0.w, s1.x, s1.y};
        const float av[3] = {s1.z, s1.w, s2.x}, ca[3] = {s2.y, s2.z, s2.w};
        float U[3], V[3], A, B, C0 = 0.0f;
        Geo GA = g;
        if (p == 0) {   // T at constant Pg: dKLIN, du/dT = -u/(2T), da/dT
          const float4 s3 = lds4(su + 3 * nthr), s4 = lds4(su + 4 * nthr);
          const float avu[3] = {s3.x, s3.y, s3.z}, cau[3] = {s3.w, s4.x, s4.y};
#pragma unroll
          for (int t = 0; t < 3; ++t) {
            U[t] = fmaf(ca[t], ddt, -avu[t] * halfT);
            V[t] = fmaf(av[t], ddt, cau[t] * halfT);
          }
          A = dkt;
          B = kldz;
          C0 = row[dkoff];
        } else if (p == 1) {   // Pg at constant T: dKLIN and da/dPg
#pragma unroll
          for (int t = 0; t < 3; ++t) {
            U[t] = ca[t];
            V[t] = av[t];
          }
          A = dkp;
          B = kldz * ddp;
          C0 = row[dkoff + 1];
        } else if (p < 5) {   // B_i: geometry factors and the shift term du/dB
          const float4 s4 = lds4(su + 4 * nthr), s5 = lds4(su + 5 * nthr);
          U[0] = s4.z; U[1] = s4.w; U[2] = s5.x;
          V[0] = -s5.y; V[1] = -s5.z; V[2] = -s5.w;
          const float* dg = row + dgoff + 5 * (p - 2);
          GA = Geo{dg[0], dg[1], dg[2], dg[3], dg[4]};
          A = kldz;
          B = kldz * (idd * row[dboff + p - 2]);
        } else {   // v_z: du/dv = lu_duv / Doppler width
#pragma unroll
          for (int t = 0; t < 3; ++t) {
            U[t] = av[t];
            V[t] = -ca[t];
          }
          A = 0.0f;
          B = kldz * P.lu_duv[lb] * idd;
        }
        float dt[7], ta[7], tb[7];
        lmap(GA, hh, ff, ta);
        lmap(g, U, V, tb);
#pragma unroll
        for (int x = 0; x < 7; ++x) dt[x] = A != 0.0f ? fmaf(A, ta[x], B * tb[x]) : B * tb[x];
        dt[0] = C0 + dt[0];
        float rfp[4] = {0.f, 0.f, 0.f, 0.f};
        if (fin) {
          if (HE && p == 2) {
            const float wout[4] = {n0 - S, n1, n2, n3};
            evol_w(es, O, wout, v);
          }
          evol_dir(es, v, dt, rfp);
        }
        if (p == 0) {
          // source-function term (1 - O) e0 dS/dT, then the HE global term
          rfp[0] = fmaf(om0, dS, rfp[0]);
          rfp[1] = fmaf(-O[4], dS, rfp[1]);
          rfp[2] = fmaf(-O[8], dS, rfp[2]);
          rfp[3] = fmaf(-O[12], dS, rfp[3]);
          if (HE) {
#pragma unroll
            for (int i = 0; i < 4; ++i) rfp[i] = fmaf(ck, OH[i], rfp[i]);
          }
        }
        if (HE && p == 1) {
#pragma unroll
          for (int i = 0; i < 4; ++i) H[i] = prop ? fmaf(rfp[i], pgk, OH[i]) : H[i];
        }
        if (FULL) {
          const int nw = P.numw;
#pragma unroll
          for (int c = 0; c < 4; ++c) jcol[((size_t)p * nz + k) * fstride + c * nw + l] = rfp[c];
        } else {
          const int j0 = C.n0[p], j1 = j0 + C.nj[p];
          for (int j = j0; j < j1; ++j) {
            float* d = Dacc + (j * 4) * nthr + l;
            const float d0 = d[0], d1 = d[nthr], d2 = d[2 * nthr], d3 = d[3 * nthr];
            const float cj = ckr[j];
            d[0] = fmaf(cj, rfp[0], fmaf(O[0], d0, fmaf(O[1], d1, fmaf(O[2], d2, O[3] * d3))));
            d[nthr] = fmaf(cj, rfp[1], fmaf(O[4], d0, fmaf(O[5], d1, fmaf(O[6], d2, O[7] * d3))));
            d[2 * nthr] = fmaf(cj, rfp[2], fmaf(O[8], d0, fmaf(O[9], d1, fmaf(O[10], d2, O[11] * d3))));
            d[3 * nthr] = fmaf(cj, rfp[3], fmaf(O[12], d0, fmaf(O[13], d1, fmaf(O[14], d2, O[15] * d3))));
          }
        }
      }
      if (FULL) {
        const int nw = P.numw;
#pragma unroll
        for (int i = 0; i < 16; ++i) ocol[((size_t)k * 16 + i) * nw + l] = O[i];
      }
      I0 = n0;
      I1 = n1;
      I2 = n2;
      I3 = n3;
      continue;
    }
    float tI = row[4 + r], tQ = 0.f, tU = 0.f, tV = 0.f, rQ = 0.f, rU = 0.f, rV = 0.f;
    float dtau[NSLOT][7];
#pragma unroll
    for (int p = 0; p < NSLOT; ++p)
#pragma unroll
      for (int x = 0; x < 7; ++x) dtau[p][x] = 0.0f;
    dtau[0][0] = row[dkoff];
    dtau[1][0] = row[dkoff + 1];
    for (int b = 0; b < nb; ++b) {
      const float* qq = row + loff + 4 * (lb + b);
      const float kldz = qq[0], a = qq[1], idd = qq[2];
      const float x0 = lp.wave + qq[3];
      // per-type sums: value (h, f) and the derivative sums of WDEV
      float hh[3] = {0, 0, 0}, ff[3] = {0, 0, 0}, av[3] = {0, 0, 0}, ca[3] = {0, 0, 0};
      float avu[3] = {0, 0, 0}, cau[3] = {0, 0, 0}, avs[3] = {0, 0, 0}, cas[3] = {0, 0, 0};
      int c = P.lu_c0[lb + b];
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const int e = c + P.lu_nt[lb + b][t];
        for (; c < e; ++c) {
          const float shf = P.comp_shift[c], st = P.comp_str[c];
          const float u = fmaf(shf, B, x0) * idd;
          float h, f;
          voigt_f32(a, u, h, f);
          const float dhv = 2.0f * fmaf(a, f, -u * h);                       // 2(-u H + a F)
          const float dha = 2.0f * (fmaf(a, h, u * f) - 0.56418958354775628f);  // 2(-1/sqrt(pi) + a H + u F)
          hh[t] = fmaf(st, h, hh[t]);
          ff[t] = fmaf(st, f, ff[t]);
          const float sv = st * dhv, sa = st * dha;
          av[t] += sv;
          ca[t] += sa;
          avu[t] = fmaf(sv, u, avu[t]);
          cau[t] = fmaf(sa, u, cau[t]);
          avs[t] = fmaf(sv, shf, avs[t]);
          cas[t] = fmaf(sa, shf, cas[t]);
        }
      }
      {
        // value part: same expressions as k_synth
        const float hs = hh[0] + hh[2], fs = ff[0] + ff[2];
        const float hl = 0.5f * hh[1] - 0.25f * hs, fl = 0.5f * ff[1] - 0.25f * fs;
        tI = fmaf(kldz, g.g1 * hs + g.g2 * hh[1], tI);
        tQ = fmaf(kldz, g.g3 * hl, tQ);
        tU = fmaf(kldz, g.g4 * hl, tU);
        tV = fmaf(kldz, g.g5 * (hh[0] - hh[2]), tV);
        rQ = fmaf(kldz, g.g3 * fl, rQ);
        rU = fmaf(kldz, g.g4 * fl, rU);
        rV = fmaf(kldz, g.g5 * (ff[0] - ff[2]), rV);
      }
      const float* dl = row + dloff + 4 * (lb + b);
      const float dkt = dl[0], dkp = dl[1], ddt = dl[2], ddp = dl[3];
      float base[7], tmp[7];
      lmap(g, hh, ff, base);
      // T at constant Pg: dKLIN, du/dT = -u/(2T), da/dT
      {
        float xe[3], xr[3];
#pragma unroll
        for (int t = 0; t < 3; ++t) {
          xe[t] = fmaf(ca[t], ddt, -avu[t] * halfT);
          xr[t] = fmaf(av[t], ddt, cau[t] * halfT);
        }
        lmap(g, xe, xr, tmp);
#pragma unroll
        for (int x = 0; x < 7; ++x) dtau[0][x] += fmaf(dkt, base[x], kldz * tmp[x]);
      }
      // Pg at constant T: dKLIN and da/dPg (the reference's KLIN*acc*DDAMDPG_TEMP)
      lmap(g, ca, av, tmp);
#pragma unroll
      for (int x = 0; x < 7; ++x) dtau[1][x] += fmaf(dkp, base[x], kldz * ddp * tmp[x]);
      // v_z: du/dv = lu_duv / Doppler width
      {
        float nca[3] = {-ca[0], -ca[1], -ca[2]};
        lmap(g, av, nca, tmp);
        const float kv = kldz * P.lu_duv[lb + b] * idd;
#pragma unroll
        for (int x = 0; x < 7; ++x) dtau[5][x] += kv * tmp[x];
      }
      // B_i: geometry factors and the shift term du/dB = shift / Doppler width
      {
        float ncs[3] = {-cas[0], -cas[1], -cas[2]};
        float sh7[7];
        lmap(g, avs, ncs, sh7);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const float* dg = row + dgoff + 5 * i;
          const Geo gd{dg[0], dg[1], dg[2], dg[3], dg[4]};
          lmap(gd, hh, ff, tmp);
          const float kb = idd * row[dboff + i];
#pragma unroll
          for (int x = 0; x < 7; ++x) dtau[2 + i][x] += kldz * fmaf(kb, sh7[x], tmp[x]);
        }
      }
    }
    float O[16], om0 = 0.0f;
    EvolSt es;
    const bool fin = isfinite(tI) && isfinite(tQ) && isfinite(tU) && isfinite(tV) && isfinite(rQ) &&
                     isfinite(rU) && isfinite(rV);
    if (!fin) {
      bad = 1;
#pragma unroll
      for (int i = 0; i < 16; ++i) O[i] = (i % 5 == 0) ? 1.f : 0.f;
    } else {
      evol_state(tI, tQ, tU, tV, rQ, rU, rV, O, om0, es);
    }
    const float n0 = fmaf(om0, S, fmaf(O[0], I0, fmaf(O[1], I1, fmaf(O[2], I2, O[3] * I3))));
    const float n1 = fmaf(-O[4], S, fmaf(O[4], I0, fmaf(O[5], I1, fmaf(O[6], I2, O[7] * I3))));
    const float n2 = fmaf(-O[8], S, fmaf(O[8], I0, fmaf(O[9], I1, fmaf(O[10], I2, O[11] * I3))));
    const float n3 = fmaf(-O[12], S, fmaf(O[12], I0, fmaf(O[13], I1, fmaf(O[14], I2, O[15] * I3))));
    float rf[NSLOT][4];
    if (fin) {
      // unrolled over the parameters: the optical-depth derivatives and the
      // response vectors stay in registers (a runtime parameter index would
      // put both arrays in local memory; measured 8-13 % slower)
      EvolW wi;
      const float win[4] = {I0 - S, I1, I2, I3};
      evol_w(es, O, win, wi);
      if (HE) {
#pragma unroll
        for (int p = 0; p < 2; ++p) evol_dir(es, wi, dtau[p], rf[p]);
        EvolW wo;
        const float wout[4] = {n0 - S, n1, n2, n3};
        evol_w(es, O, wout, wo);
#pragma unroll
        for (int p = 2; p < NSLOT; ++p) evol_dir(es, wo, dtau[p], rf[p]);
      } else {
#pragma unroll
        for (int p = 0; p < NSLOT; ++p) evol_dir(es, wi, dtau[p], rf[p]);
      }
    } else {
#pragma unroll
      for (int p = 0; p < NSLOT; ++p)
#pragma unroll
        for (int c = 0; c < 4; ++c) rf[p][c] = 0.0f;
    }
    // source-function term of the T response: (1 - O) e0 dS/dT, with
    // dS/dT = c1 (c2/T^2) e^q / (e^q - 1)^2 (src/rtesolver.f90:1039-1066)
    {
      const float dS = lp.c1 * (q / T) * ((em1 + 1.0f) / (em1 * em1));
      rf[0][0] = fmaf(om0, dS, rf[0][0]);
      rf[0][1] = fmaf(-O[4], dS, rf[0][1]);
      rf[0][2] = fmaf(-O[8], dS, rf[0][2]);
      rf[0][3] = fmaf(-O[12], dS, rf[0][3]);
    }
    if (HE) {
      const float ck = row[heoff], pgk = row[heoff + 1];
      const bool prop = O[0] > 1.0e-5f;
      float OH[4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
        OH[i] = prop ? O[4 * i] * H[0] + O[4 * i + 1] * H[1] + O[4 * i + 2] * H[2] + O[4 * i + 3] * H[3] : H[i];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        rf[0][i] = fmaf(ck, OH[i], rf[0][i]);
        H[i] = prop ? fmaf(rf[1][i], pgk, OH[i]) : H[i];
      }
    }
    if (FULL) {
      const int nw = P.numw;
#pragma unroll
      for (int p = 0; p < NSLOT; ++p)
#pragma unroll
        for (int c = 0; c < 4; ++c) jcol[((size_t)p * nz + k) * fstride + c * nw + l] = rf[p][c];
#pragma unroll
      for (int i = 0; i < 16; ++i) ocol[((size_t)k * 16 + i) * nw + l] = O[i];
      I0 = n0;
      I1 = n1;
      I2 = n2;
      I3 = n3;
      continue;
    }
    // node accumulation
    const float* ck = coef + k * np;
#pragma unroll
    for (int p = 0; p < NSLOT; ++p) {
      const int j0 = C.n0[p], j1 = j0 + C.nj[p];
      for (int j = j0; j < j1; ++j) {
        float* d = Dacc + (j * 4) * nthr + l;
        const float d0 = d[0], d1 = d[nthr], d2 = d[2 * nthr], d3 = d[3 * nthr];
        const float cj = ck[j];
        d[0] = fmaf(cj, rf[p][0], fmaf(O[0], d0, fmaf(O[1], d1, fmaf(O[2], d2, O[3] * d3))));
        d[nthr] = fmaf(cj, rf[p][1], fmaf(O[4], d0, fmaf(O[5], d1, fmaf(O[6], d2, O[7] * d3))));
        d[2 * nthr] = fmaf(cj, rf[p][2], fmaf(O[8], d0, fmaf(O[9], d1, fmaf(O[10], d2, O[11] * d3))));
        d[3 * nthr] = fmaf(cj, rf[p][3], fmaf(O[12], d0, fmaf(O[13], d1, fmaf(O[14], d2, O[15] * d3))));
      }
    }
    I0 = n0;
    I1 = n1;
    I2 = n2;
    I3 = n3;
  }
  const int nw = P.numw;
  const int nfreq = 4 * nw;
  unsigned mask[2] = {0u, 0u};
  if (active) {
    double* o = syn + (size_t)col * 4 * nw;
    o[0 * nw + l] = (double)I0 * (double)gain[4 * l + 0];
    o[1 * nw + l] = (double)I1 * (double)gain[4 * l + 1];
    o[2 * nw + l] = (double)I2 * (double)gain[4 * l + 2];
    o[3 * nw + l] = (double)I3 * (double)gain[4 * l + 3];
    if (!(isfinite(I0) && isfinite(I1) && isfinite(I2) && isfinite(I3))) bad = 1;
  }
  if (FULL) {
    if (status && __any_sync(__activemask(), bad) && (l & 31) == 0) atomicOr(&status[col], FZ_NAN);
    return;
  }
  if (active) {
    // EQVDSYN = REAL(sum) * GAIN (src/forward.f90:614-621)
    float* jo = jac + (size_t)col * np * nfreq;
    for (int j = 0; j < np; ++j)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float v = Dacc[(j * 4 + c) * nthr + l] * gain[4 * l + c];
        jo[(size_t)j * nfreq + c * nw + l] = v;
        if (isinf(v)) mask[j >> 5] |= 1u << (j & 31);
      }
  }
  // columns whose |.| sum overflows REAL*4 are zeroed (:673-679)
  if (mask[0]) atomicOr(&inf_mask[0], mask[0]);
  if (mask[1]) atomicOr(&inf_mask[1], mask[1]);
  __syncthreads();
  if ((inf_mask[0] | inf_mask[1]) && active) {
    float* jo = jac + (size_t)col * np * nfreq;
    for (int j = 0; j < np; ++j)
      if (inf_mask[j >> 5] & (1u << (j & 31)))
#pragma unroll
        for (int c = 0; c < 4; ++c) jo[(size_t)j * nfreq + c * nw + l] = 0.0f;
  }
  if (status && __any_sync(__activemask(), bad) && (l & 31) == 0) atomicOr(&status[col], FZ_NAN);
}

// k_synth_rf with the block-size bound its thread count needs
template <bool HE, bool FULL, typename... A>
void launch_synth_rf(bool blend, int blocks, int threads, size_t sms, cudaStream_t s, A... a) {
  if (threads <= 256) {
    if (blend)
      k_synth_rf<HE, FULL, 256, true><<<blocks, threads, sms, s>>>(a...);
    else
      k_synth_rf<HE, FULL, 256, false><<<blocks, threads, sms, s>>>(a...);
  } else {
    if (blend)
      k_synth_rf<HE, FULL, 512, true><<<blocks, threads, sms, s>>>(a...);
    else
      k_synth_rf<HE, FULL, 512, false><<<blocks, threads, sms, s>>>(a...);
  }
}

template <bool HE, bool FULL>
cudaError_t set_synth_rf_attr(cudaFuncAttribute attr, int v) {
  cudaError_t e = cudaFuncSetAttribute(k_synth_rf<HE, FULL, 256, false>, attr, v);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_rf<HE, FULL, 512, false>, attr, v);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_synth_rf<HE, FULL, 256, true>, attr, v);
  return e == cudaSuccess ? cudaFuncSetAttribute(k_synth_rf<HE, FULL, 512, true>, attr, v) : e;
}

// true when some region of the context holds blended lines
bool has_blends(const fz_ctx* c);

// Response functions at emergence from the local ones (FULL mode of
// k_synth_rf): RF(K) = O_NZ ... O_{K+1} RF_loc(K), OLD_DSYN_PROPAGATION
// (src/forward.f90:511-548), times GAIN as CALCULATE_EQUIVALENT_DSYN with
// NJ = NZ (:604-621).  One CTA per column, one thread per wavelength walking
// down from the top with the 4x4 product of the operators above in
// registers; in place on rf.  A (parameter, height) column with an infinite
// entry is zeroed, the SUM(ABS(.)) > HUGE test of :672-679.
__global__ void __launch_bounds__(512) k_rf_prop(int nz, int nw, const float* __restrict__ gain,
                                                 const float* __restrict__ oscr, float* __restrict__ rf,
                                                 const int* __restrict__ list = nullptr,
                                                 const int* __restrict__ nlist = nullptr) {
  extern __shared__ int flg[];
  if (list && (int)blockIdx.x >= *nlist) return;
  const int col = list ? list[blockIdx.x] : (int)blockIdx.x, l = threadIdx.x;
  for (int i = l; i < nz; i += blockDim.x) flg[i] = 0;
  __syncthreads();
  const bool active = l < nw;
  const size_t nfreq = 4 * (size_t)nw;
  float* base = rf + (size_t)col * NSLOT * nz * nfreq + l;
  if (active) {
    float g[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) g[c] = gain[4 * l + c];
    const float* ob = oscr + (size_t)col * nz * 16 * nw + l;
    float A[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) A[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    for (int k = nz - 1; k >= 0; --k) {
      int f = 0;
#pragma unroll
      for (int p = 0; p < NSLOT; ++p) {
        float* q = base + ((size_t)p * nz + k) * nfreq;
        const float r0 = q[0], r1 = q[nw], r2 = q[2 * nw], r3 = q[3 * nw];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float v = fmaf(A[4 * i], r0, fmaf(A[4 * i + 1], r1, fmaf(A[4 * i + 2], r2, A[4 * i + 3] * r3))) * g[i];
          q[(size_t)i * nw] = v;
          if (isinf(v)) f |= 1 << p;
        }
      }
      if (f) atomicOr(&flg[k], f);
      float O[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) O[i] = ob[((size_t)k * 16 + i) * nw];
      float B[16];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          B[4 * i + j] = fmaf(A[4 * i], O[j], fmaf(A[4 * i + 1], O[4 + j], fmaf(A[4 * i + 2], O[8 + j], A[4 * i + 3] * O[12 + j])));
#pragma unroll
      for (int i = 0; i < 16; ++i) A[i] = B[i];
    }
  }
  __syncthreads();
  if (active)
    for (int k = 0; k < nz; ++k) {
      const int f = flg[k];
      if (!f) continue;
      for (int p = 0; p < NSLOT; ++p)
        if (f & (1 << p))
#pragma unroll
          for (int c = 0; c < 4; ++c) base[((size_t)p * nz + k) * nfreq + (size_t)c * nw] = 0.0f;
    }
}

}  // namespace

#include "fz_lm.cuh"
#include "fz_lm_big.cuh"

namespace {

// ------------------------------------------------------------------ k_gain
// HSRA continuum normalisation, src/normalization.f90:696-754: one block;
// warp 0 runs the chemistry of the 387 layers (nelec chain), then every
// thread integrates its wavelengths through the continuum-only atmosphere
// with the reference's REAL*4 rounding of the intermediate intensities.
__global__ void k_gain(const DevParams* __restrict__ Pg, const Consts* __restrict__ Kg,
                       const PFTable* __restrict__ tb, const double* __restrict__ lam_l /* (numw) [A] */, float* gain,
                       int* status) {
  extern __shared__ double sm_gain[];   // (387 x nreg) continuum opacities
  const DevParams& P = *Pg;
  const Consts& K = *Kg;
  const int N = FZ_HSRA_LEN;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    double ab[3];
    for (int j = 0; j < 3; ++j) ab[j] = K.lane_elem[32 * j + lane] >= 0 ? K.ab10[K.lane_elem[32 * j + lane]] : 0.0;
    double nelec = 0.0;
    WarpSaha w;
    int st = 0;
    for (int k = 0; k < N; ++k) {
      const double T = (double)fz_tab_hsra_tem[k];
      saha_prepare(w, T, K, tb, lane);
      const RhoOut r = get_rho_warp(w, ab, (double)fz_tab_hsra_pg[k], nelec, K, lane);
      st |= r.status;
      if (lane < P.nreg) sm_gain[k * P.nreg + lane] = opac_continuum(T, nelec, r.nhyd, P.cont[lane]);
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

// The same independent FMA chains in FP64: the FP64 pipe's peak.
__global__ void k_fp64_peak(double* out, int iters, double s) {
  double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9;
  double a4 = a0 + 4e-9, a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
  const double m = 0.999999999;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      a0 = fma(a0, m, s); a1 = fma(a1, m, s); a2 = fma(a2, m, s); a3 = fma(a3, m, s);
      a4 = fma(a4, m, s); a5 = fma(a5, m, s); a6 = fma(a6, m, s); a7 = fma(a7, m, s);
    }
  }
  const double r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (r == 1234.5) out[0] = r;
}

// ------------------------------------------------------------------ context
const double kAbund[FZ_NELEM] = {
#include "fz_abund.inc"
};
const double kMatom[FZ_NELEM] = {
#include "fz_matom.inc"
};
const double kXI[FZ_NELEM] = {
#include "fz_xi.inc"
};
const double kXII[FZ_NELEM] = {
#include "fz_xii.inc"
};

void host_consts(Consts& K) {
  K.csaha1 = std::pow(HPLA, 3.0) / std::pow(2.0 * DPI * MELE * KBOL, 3.0 / 2.0);
  K.csaha2 = EVOLT / KBOL;
  K.rbohr = std::pow(HPLA, 2.0) / (4.0 * std::pow(DPI, 2.0) * MELE * std::pow(QELE, 2.0));
  K.deno_sa = 0.0;
  K.deno_sam = 0.0;
  for (int i = 0; i < FZ_NELEM; ++i) {
    K.ab10[i] = std::pow(10.0, kAbund[i] - 12.0);
    K.deno_sa = K.deno_sa + K.ab10[i];
  }
  for (int i = 0; i < FZ_NELEM; ++i) K.deno_sam = K.deno_sam + MAMU * kMatom[i] * K.ab10[i];
  // lane/slot assignment of the elements: exponential-form elements first
  std::vector<int> order;
  PFTable* t = new PFTable;
  fzh_pf_table(t);
  for (int pass = 0; pass < 2; ++pass)
    for (int e = 0; e < FZ_NELEM; ++e) {
      bool ex = false;
      for (int s = 0; s < 3; ++s)
        for (int i = 0; i < t->nv[e][s]; ++i) ex = ex || t->p[e][s][i].form == 1;
      if (ex == (pass == 0)) order.push_back(e);
    }
  delete t;
  for (int i = 0; i < 96; ++i) K.lane_elem[i] = i < (int)order.size() ? order[i] : -1;
}

// Wavelength-only factors of OPAC_CONTINUUM at lambda0 [A], src/cont_opacity.f90:48-357.
ContP host_cont(double l0) {
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
  ContP c;
  std::memset(&c, 0, sizeof(c));
  const double lm = l0 / 1e4;
  const double p2 = std::pow(lm, 2.0), p3 = std::pow(lm, 3.0), p4 = std::pow(lm, 4.0);
  if (lm < 0.3645) {
    c.nff = 4;
    for (int i = 0; i < 4; ++i) c.ffc[i] = A2[i] * p2 + B2[i] + C2[i] / lm + D2[i] / p2 + E2[i] / p3 + F2[i] / p4;
  } else {
    c.nff = 6;
    for (int i = 0; i < 6; ++i) c.ffc[i] = A1[i] * p2 + B1[i] + C1[i] / lm + D1[i] / p2 + E1[i] / p3 + F1[i] / p4;
  }
  const double LAMBDAP = 1.6419, CTE = 0.75e-18, ALPHA = (HPLA * LIGHT / KBOL) * 1e4;
  static const double CC[6] = {152.519, 49.534, -118.858, 92.536, -34.194, 4.982};
  if (lm < LAMBDAP) {
    const double com = 1.0 / lm - 1.0 / LAMBDAP;
    double sg = CC[0] + CC[1] * std::pow(com, 0.5) + CC[2] * com + CC[3] * std::pow(com, 1.5) +
                CC[4] * std::pow(com, 2.0) + CC[5] * std::pow(com, 2.5);
    c.sbf = CTE * sg * std::pow(lm, 3.0) * std::pow(com, 1.5);
    c.bfa1 = ALPHA / LAMBDAP;
    c.bfa2 = ALPHA / lm;
  }
  const double IOPOT = (double)13.595f, E8 = (double)1e-8f;   // REAL*4 literals, :255-264
  const double HC1 = E8 * IOPOT * EVOLT / (HPLA * LIGHT);
  const double HC2 = std::pow(E8, 3.0) * 64.0 * std::pow(DPI, 4.0) * MELE * std::pow(QELE, 10.0) /
                     (3.0 * std::sqrt(3.0) * std::pow(LIGHT, 4.0) * std::pow(HPLA, 6.0));
  const double HC3 = HPLA * LIGHT / (KBOL * E8);
  const double HC4 = IOPOT * EVOLT / KBOL;
  c.n0 = 1 + (int)std::floor(std::sqrt(HC1 * l0));
  c.hpre = HC2 * std::pow(l0, 3.0);
  c.c3l = HC3 / l0;
  c.c4 = HC4;
  c.ray = (5.799e-13 + (1.422e-6 + 2.784 / std::pow(l0, 2.0)) / std::pow(l0, 2.0)) / std::pow(l0, 4.0);
  c.ct = (8.0 * DPI / 3.0) * (std::pow(QELE / LIGHT, 4.0)) / std::pow(MELE, 2.0);
  return c;
}

// REFRAX, src/atom_database.f90:1039-1074
double host_refrax(double w) {
  const double T = 15.0, P = 760.0, H = 0.0;
  const double s = 1.0 / std::pow(w, 2.0);
  const double r = 6.4328e-5 + 2.94981e-2 / (146.0 - s) + 2.554e-4 / (41.0 - s);
  const double y = 1.0 / (273.15 + T);
  const double alpha = 3.67e-3 + 3.3e-4 * std::exp((0.19 - w) / 0.12);
  const double wvsp = std::pow(
      10.0, -55.1132754 +
                y * (1.19551822e5 +
                     y * (-9.70108858e7 + y * (4.12856913e10 + y * (-9.87931835e12 + y * (1.25868645e15 - 6.66885272e16 * y))))));
  const double wvp = 1.0e-2 * H * wvsp;
  return 1.0 + 1.31579e-3 * r * P / (1.0 + alpha * (T - 1.0) / (1.0 + 15.0 * alpha)) - 5.49e-8 * wvp / (1.0 + alpha * T);
}

// Per-line constants of OPAC_LINE (src/line_opacity.f90:34-108) and
// GET_DAMPING (src/damping.f90:842-1012; ABO or Unsold van der Waals).
LineP host_line(const fz_line& L, double wdif, const Consts& K) {
  LineP q;
  std::memset(&q, 0, sizeof(q));
  const int z = L.zn - 1;
  const double m = kMatom[z];
  q.l0 = L.l0;
  q.wdif = wdif;
  q.zn = L.zn;
  q.ion = L.ion;
  q.term1 = std::sqrt(DPI) * std::pow(QELE, 2.0) / (MELE * LIGHT) * std::pow(10.0, L.loggf) * L.l0 * 1e-8;
  q.m2k = m * MAMU / (2.0 * KBOL);
  q.chik = L.eplow * EVOLT / KBOL;
  q.hclk = HPLA * LIGHT / (1.0e-8 * L.l0 * KBOL);
  q.nab = std::pow(10.0, kAbund[z] - 12.0);
  q.xi_k = K.csaha2 * kXI[z];
  q.xii_k = K.csaha2 * kXII[z];
  q.vdk = 2.0 * KBOL / (MAMU * m);
  const double lambda = L.l0 * 1e-8;
  q.grad = 0.2223 / std::pow(lambda, 2.0);
  q.dfac = lambda / (4.0 * DPI);
  const double mu_h = MAMU * (m * kMatom[0]) / (m + kMatom[0]);
  const double mu_he = MAMU * (m * kMatom[1]) / (m + kMatom[1]);
  const double he = std::pow(10.0, kAbund[1] - 12.0);
  if (L.sigma > 0 && L.alpha > 0) {
    const double e1 = 2.0 - L.alpha / 2.0, e2 = (1.0 - L.alpha) / 2.0;
    const double gf =
        1.0 + (-0.5748646 + (0.9512363 + (-0.6998588 + (0.4245549 - 0.1010678 * e1) * e1) * e1) * e1) * e1;
    double beta = std::pow(4.0 / DPI, L.alpha / 2.0) * gf * std::pow(1e6, L.alpha) * (L.sigma * std::pow(K.rbohr, 2.0)) *
                  std::pow(8.0 * KBOL / DPI, e2);
    beta = 2.0 * beta;
    q.gc = beta * (std::pow(mu_h, -e2) + (double)0.3181818f * he * std::pow(mu_he, -e2));
    q.ge = e2;
  } else {
    double rindex = (double)1.0004f;
    if (lambda * 1e8 >= 1800.0) rindex = host_refrax(lambda * 1e4);
    const double lvac = rindex * lambda;
    const double epupp = L.eplow + (HPLA * LIGHT / lvac) / EVOLT;
    const double ionf = (double)(float)(L.ion - 1);
    double ed1, ed2, chyd;
    if (L.ion == 1) {
      ed1 = std::max(kXI[z] - epupp - kXI[z] * ionf, 1.0);
      ed2 = std::max(kXI[z] - L.eplow - kXI[z] * ionf, 3.0);
      chyd = 1.0;
    } else {
      ed1 = std::max(kXII[z] - epupp - kXI[z] * ionf, 1.0);
      ed2 = std::max(kXII[z] - L.eplow - kXI[z] * ionf, 3.0);
      chyd = (double)1.741f;
    }
    chyd = chyd * 17.0 * std::pow(8.0 * KBOL / DPI, 0.3);
    chyd = chyd * std::pow(std::pow(10.0, -30.5325) * (1.0 / std::pow(ed1, 2.0) - 1.0 / std::pow(ed2, 2.0)), 0.4);
    q.gc = chyd * (std::pow(mu_h, -0.3) + he * std::pow(mu_he, -0.3));
    q.ge = 0.3;
  }
  return q;
}

}  // namespace

// ----------------------------------------------------------- LSF convolution
// CALCULATE_EQUIVALENT_SYN1D / CALCULATE_EQUIVALENT_DSYN with MLSF
// (src/forward.f90:793-853, :615-657, :736-772): every Stokes row of NUMW
// values is convolved, region by region, with the region's line spread
// function -- a circular convolution over the region's NUMWAVE points (the
// reference's real FFT pair without padding, the kernel divided by its
// length against FFTW's unnormalised inverse): out(i) = sum_j s(j)
// YK((i - j) mod n), in FP64 on the DBLE of the row, the result REAL*4.
// Regions without a valid LSF are left as they are.
struct LsfConf {
  int nreg;
  int off[MAXREG + 1];
  int valid[MAXREG];
};

// One warp per (row, region); rows of numw values, rows_per_col rows per
// column; with list, column c of the launch is column list[c] (c < *nlist).
// Dynamic shared memory: numw doubles per warp.
template <typename T>
__global__ void __launch_bounds__(256) k_lsf(LsfConf L, long long nrows, int rows_per_col, int numw,
                                             const int* __restrict__ list, const int* __restrict__ nlist,
                                             const double* __restrict__ ker, T* __restrict__ data) {
  extern __shared__ double sm_lsf[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  double* sv = sm_lsf + (size_t)wib * numw;
  const long long nwork = nrows * L.nreg;
  const long long nl = list ? (long long)*nlist : 0;
  for (long long wk = (long long)blockIdx.x * wpb + wib; wk < nwork; wk += (long long)gridDim.x * wpb) {
    const int reg = (int)(wk % L.nreg);
    const long long r = wk / L.nreg;
    if (!L.valid[reg]) continue;
    long long col = r / rows_per_col;
    const int sub = (int)(r % rows_per_col);
    if (list) {
      if (col >= nl) continue;
      col = list[col];
    }
    T* row = data + ((size_t)col * rows_per_col + sub) * numw;
    const int o = L.off[reg], n = L.off[reg + 1] - o;
    for (int j = lane; j < n; j += 32) sv[j] = (double)row[o + j];
    __syncwarp();
    const double* kr = ker + o;
    for (int i = lane; i < n; i += 32) {
      double acc = 0.0;
      int ki = i;   // (i - j) mod n
      for (int j = 0; j < n; ++j) {
        acc = fma(sv[j], kr[ki], acc);
        ki = ki == 0 ? n - 1 : ki - 1;
      }
      row[o + i] = (T)(float)acc;
    }
    __syncwarp();
  }
}

constexpr int NKERN = 15;   // k_chain, k_opac, k_synth, k_opac_rf, k_synth_rf, k_lm_fill, k_lm_accept, k_lm_normal, k_lm_solve, k_lm_update, k_chemder, k_rf_prop, k_lsf, k_saha, k_chain_pre

struct fz_ctx {
  int device = 0;
  int nz = 0, numw = 0, nreg = 0, nlu = 0, sw = 0;
  std::vector<fz_line> lines;
  std::vector<fz_region> regs;
  std::vector<float> gain;   // (4, numw)
  DevParams hp{};
  DevParams* d_params = nullptr;
  Consts* d_consts = nullptr;
  PFTable* d_pf = nullptr;
  PFDTable* d_pfd = nullptr;
  struct {
    int chain_warps = 4;       // k_chain warps per block
    int chain_lanes = 0;       // k_chain lanes per column: 32, 16, or 0 = by column count
    int chemder_bpsm = 32;     // k_chemder resident-block cap per SM (0 = one block per 4 cells)
    int opacrf_threads = 256;  // k_opac_rf block size
    int lm_slots = 8192;       // pixels in flight when fz_lm_opts.slots == 0
  } tune;
  float* d_oscr = nullptr;   // operators of the full-height RF path (ncol, nz, 16, numw)
  double* d_smooth = nullptr;   // SMOOTHING_B buffers
  // LSF convolution per spectral region (LSF_INIT, src/pre_post_duties.f90:742-900):
  // kernels YK (sum 1, index 0 = centre) at the regions' offsets in d_lsf
  struct {
    bool on = false;
    int valid[MAXREG] = {};
    std::vector<double> yk;
  } lsf;
  double* d_lsf = nullptr;
  size_t smooth_len = 0;
  size_t oscr_len = 0;
  LamP* d_lam = nullptr;
  float* d_gain = nullptr;
  // scratch (grown on demand): per (column, height) nH, ne and the opacity slab
  float* d_slab = nullptr;
  double2* d_chem = nullptr;
  double2* d_saha = nullptr;   // k_saha's rows of a chunk of columns
  size_t saha_bytes = 0;
  size_t scratch_cols = 0;
  // staging for the host-buffer API
  float* d_model = nullptr;
  double* d_syn = nullptr;
  int* d_status = nullptr;
  size_t io_cols = 0;
  // staging of the host-buffer inversion (grow on demand, kept across calls)
  struct {
    double *obs = nullptr, *chi = nullptr, *syn = nullptr, *tgt = nullptr;
    float *init = nullptr, *out = nullptr;
    int *it = nullptr, *st = nullptr;
    float* fb = nullptr;   // the fallback model (13, nz)
    double* state = nullptr;   // the final LM states (5, npix), when asked for
    size_t cap = 0, state_cap = 0;
    bool has_syn = false;
  } inv;
  cudaStream_t stream = nullptr;
  int nsm = 148;
  // per-kernel profiling (pending event pairs are resolved on read)
  bool prof = false;
  struct Pending {
    int kernel;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> ev_pool;   // resolved events, reused by later scopes
  double prof_ms[NKERN] = {};
  int prof_n[NKERN] = {};
  long long prof_items[NKERN] = {};
  // response functions: node layout, hat coefficients (nz x np), RF slab
  RFConf rf{};
  RFConf* d_rf = nullptr;
  float* d_coef = nullptr;
  float* d_rfslab = nullptr;
  double4* d_chemd = nullptr;   // chemistry derivatives per (column, height)
  size_t rf_cols = 0;
  float* d_jac = nullptr;   // staging of the host-buffer API
  size_t jac_cols = 0;
  double* d_coef64 = nullptr;   // (nz, np) hat table in FP64 for the LM update
  // LM slot pool (grown on demand)
  LMSlots lm{}, lm2{};   // two pools: the tail of an inversion is compacted into the other one
  int* d_dest = nullptr;
  int* d_act = nullptr;   // the occupied slots of the pool, in order (device-driven loop)
  size_t lm_cap = 0;
  int lm_np = 0;
  LMQueue* d_q = nullptr;
  int* h_done = nullptr;
  LMQueue* h_q = nullptr;   // pinned copy of the work-queue state   // pinned
  // node layouts whose forward accumulation does not fit in shared memory:
  // the node Jacobian is contracted from the response functions at every
  // height (scratch (columns, 6, nz, NFREQ)), and the LM runs its large-NP
  // kernels with the per-node tables in device memory
  bool rf_full = false;
  float* d_rfbig = nullptr;
  size_t rfbig_len = 0;
  int* d_nrow = nullptr;       // (np) model row of each node
  double* d_nnorm = nullptr;   // (np) PARAM_NORMS of each node
  double* d_nhss = nullptr;    // (np, np) PEN_HSS of the last configured regularisation
  std::vector<double> nhss_host;
  double* d_svd = nullptr;     // per-slot SVD scratch (2 np^2)
  size_t svd_len = 0;
  float* d_wsy = nullptr;      // warm start: network outputs (npix, np), normalisation, base model
  size_t wsy_len = 0;
  float* d_wsnorm = nullptr;
  size_t wsnorm_len = 0;
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
#define FZ_CK_RC(x)                           \
  do {                                        \
    int _rc = (x);                            \
    if (_rc) return _rc;                      \
  } while (0)

// k_chain takes precomputed Saha factors (k_saha) for batches of at most
// SAHA_MAX_COLS columns: the rows of that many columns.
constexpr int SAHA_MAX_COLS = 1024;
size_t saha_row_bytes(const fz_ctx* c) { return (size_t)(2 * c->nz - 1) * 96 * sizeof(double2); }
int saha_chunk_cols(int ncol) { return std::min(ncol, SAHA_MAX_COLS); }

int ensure_scratch(fz_ctx* c, int ncol) {
  if ((size_t)ncol > c->scratch_cols) {
    cudaFree(c->d_slab);
    cudaFree(c->d_chem);
    c->d_slab = nullptr;
    c->d_chem = nullptr;
    c->scratch_cols = 0;
    FZ_CK(cudaMalloc(&c->d_slab, (size_t)ncol * c->nz * c->sw * sizeof(float)));
    FZ_CK(cudaMalloc(&c->d_chem, (size_t)ncol * c->nz * sizeof(double2)));
    c->scratch_cols = ncol;
  }
  const size_t sb = (size_t)saha_chunk_cols(ncol) * saha_row_bytes(c);
  if (sb > c->saha_bytes) {
    cudaFree(c->d_saha);
    c->d_saha = nullptr;
    c->saha_bytes = 0;
    FZ_CK(cudaMalloc(&c->d_saha, sb));
    c->saha_bytes = sb;
    // k_saha's shared memory (the samples' temperatures and terms) above the
    // default 48 KB for tall columns; set here, before any stream capture
    const size_t ssm = saha_smem(c->nz);
    if (ssm > 48 * 1024 && ssm <= 200 * 1024) {
      FZ_CK(cudaFuncSetAttribute(k_saha<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm));
      FZ_CK(cudaFuncSetAttribute(k_saha<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm));
    }
  }
  return 0;
}

// brackets one launch with events; `items` = columns (or slots) it processes
bool has_blends(const fz_ctx* c) {
  for (const fz_region& r : c->regs)
    if (r.nblend > 1) return true;
  return false;
}

struct ProfScope {
  fz_ctx* c;
  int kernel;
  cudaStream_t s;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(fz_ctx* c_, int k, cudaStream_t s_, long long items = 0) : c(c_), kernel(k), s(s_) {
    if (!c->prof) return;
    c->prof_items[k] += items;
    a = take();
    b = take();
    cudaEventRecord(a, s);
  }
  cudaEvent_t take() {
    if (c->ev_pool.empty()) {
      cudaEvent_t e = nullptr;
      cudaEventCreate(&e);
      return e;
    }
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  ~ProfScope() {
    if (!c->prof) return;
    cudaEventRecord(b, s);
    c->pending.push_back({kernel, a, b});
  }
};

// k_chain with wpb warps per block and lanes (32 or 16) lanes per column;
// lanes = 0 picks 16 when the batch fills 8 warps per SM with two columns a
// warp (throughput: half the warp instructions per column) and 32 below
// (latency: every column's chain gets a warp of its own).  chem: the (nH, ne)
// scratch of the batch, the context's own buffer when null.
void launch_k_chain(fz_ctx* c, int ncol, const float* d_model, float* d_mout, int* d_status, int hydrostatic, int wpb,
                    int lanes, cudaStream_t s, double2* chem = nullptr, const int* list = nullptr,
                    const int* nlist = nullptr, bool pre = true) {
  if (!chem) chem = c->d_chem;
  if (hydrostatic == 2) {   // HE anchored at log tau5 ~ 0 (HYDRO_TOP off)
    ProfScope ps(c, 0, s, ncol);
    const dim3 g((unsigned)(((size_t)ncol * 32 + 127) / 128));
    k_chain_med<<<g, 128, 0, s>>>(c->d_consts, c->d_pf, ncol, c->nz, d_model, d_mout, chem, d_status);
    return;
  }
  if (lanes != 16 && lanes != 32) lanes = ncol >= 16 * c->nsm ? 16 : 32;
  const int nsamp = hydrostatic ? 2 * c->nz - 1 : c->nz;
  // the precomputed form when the context's rows hold the batch's first
  // SAHA_MAX_COLS columns and k_saha's shared memory fits; a batch of known
  // size takes one form, a listed batch (count on the device) launches both,
  // each gated by the count
  const int per = saha_chunk_cols(ncol);
  const size_t ssm = saha_smem(c->nz);
  pre = pre && c->d_saha && (size_t)per * nsamp * 96 * sizeof(double2) <= c->saha_bytes && ssm <= 200 * 1024;
  const bool plain = !pre || list || ncol > SAHA_MAX_COLS;
  const bool fast = pre && (list || ncol <= SAHA_MAX_COLS);
  const int gate = list ? SAHA_MAX_COLS : 0;
  if (plain) {
    ProfScope ps(c, 0, s, ncol);
    const size_t threads = (size_t)ncol * lanes;
    const dim3 gc((unsigned)((threads + wpb * 32 - 1) / (wpb * 32)));
    const int pg = fast ? -gate : 0;
    if (lanes == 16) {
      if (hydrostatic)
        k_chain<true, 16, false><<<gc, wpb * 32, 0, s>>>(c->d_consts, c->d_pf, ncol, c->nz, d_model, d_mout, chem,
                                                         d_status, list, nlist, nullptr, 0, 0, pg);
      else
        k_chain<false, 16, false><<<gc, wpb * 32, 0, s>>>(c->d_consts, c->d_pf, ncol, c->nz, d_model, d_mout, chem,
                                                          d_status, list, nlist, nullptr, 0, 0, pg);
    } else {
      if (hydrostatic)
        k_chain<true, 32, false><<<gc, wpb * 32, 0, s>>>(c->d_consts, c->d_pf, ncol, c->nz, d_model, d_mout, chem,
                                                         d_status, list, nlist, nullptr, 0, 0, pg);
      else
        k_chain<false, 32, false><<<gc, wpb * 32, 0, s>>>(c->d_consts, c->d_pf, ncol, c->nz, d_model, d_mout, chem,
                                                          d_status, list, nlist, nullptr, 0, 0, pg);
    }
  }
  if (!fast) return;
  // the small-batch form: every column's Saha rows (split over a few CTAs a
  // column, for latency), then the chains on them, always 32 lanes a column
  const int cn = per;
  {
    ProfScope ps(c, 13, s, list ? 0 : cn);
    const dim3 gs((unsigned)cn, cn <= c->nsm ? 4u : 1u);
    if (hydrostatic)
      k_saha<true><<<gs, 256, ssm, s>>>(c->d_consts, c->d_pf, ncol, c->nz, d_model, c->d_saha, 0, cn, list, nlist,
                                        gate);
    else
      k_saha<false><<<gs, 256, ssm, s>>>(c->d_consts, c->d_pf, ncol, c->nz, d_model, c->d_saha, 0, cn, list, nlist,
                                         gate);
  }
  ProfScope ps(c, 14, s, list ? 0 : cn);
  const dim3 gc((unsigned)(((size_t)cn * 32 + wpb * 32 - 1) / (wpb * 32)));
  if (hydrostatic)
    k_chain<true, 32, true><<<gc, wpb * 32, 0, s>>>(c->d_consts, c->d_pf, ncol, c->nz, d_model, d_mout, chem,
                                                    d_status, list, nlist, c->d_saha, 0, cn, gate);
  else
    k_chain<false, 32, true><<<gc, wpb * 32, 0, s>>>(c->d_consts, c->d_pf, ncol, c->nz, d_model, d_mout, chem,
                                                     d_status, list, nlist, c->d_saha, 0, cn, gate);
}

// The LSF pass over nrows rows of numw values (no-op without a valid LSF).
template <typename T>
int launch_lsf(fz_ctx* c, T* d_data, long long nrows, int rows_per_col, cudaStream_t s, const int* list = nullptr,
               const int* nlist = nullptr) {
  if (!c->lsf.on || nrows <= 0) return 0;
  LsfConf L{};
  L.nreg = c->nreg;
  for (int r = 0; r < c->nreg; ++r) {
    L.off[r + 1] = L.off[r] + c->regs[r].numwave;
    L.valid[r] = c->lsf.valid[r];
  }
  const size_t smem = (size_t)8 * c->numw * sizeof(double);
  if (smem > 227 * 1024) return FZ_ERR_LIMIT;
  if (smem > 48 * 1024) FZ_CK(cudaFuncSetAttribute(k_lsf<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long work = nrows * c->nreg;
  const int blocks = (int)std::min<long long>((work + 7) / 8, (long long)c->nsm * 16);
  {
    ProfScope ps(c, 12, s, list ? 0 : (nrows / rows_per_col));
    k_lsf<T><<<blocks, 256, smem, s>>>(L, nrows, rows_per_col, c->numw, list, nlist, c->d_lsf, d_data);
  }
  return cuda_fail(cudaGetLastError());
}

// The synthesis of ncol columns, or with a list of the columns list[0,
// *nlist) among ncol slots (an inversion pool's occupied slots; the count
// read on the device, so that a captured graph replays for any count).
int launch_forward(fz_ctx* c, int ncol, const float* d_model, int hydrostatic, double* d_syn, float* d_mout,
                   int* d_status, cudaStream_t s, const int* list = nullptr, const int* nlist = nullptr) {
  int rc = ensure_scratch(c, ncol);
  if (rc) return rc;
  if (d_status) FZ_CK(cudaMemsetAsync(d_status, 0, ncol * sizeof(int), s));
  launch_k_chain(c, ncol, d_model, d_mout, d_status, hydrostatic, c->tune.chain_warps, c->tune.chain_lanes, s,
                 nullptr, list, nlist);
  FZ_CK(cudaGetLastError());
  {
    ProfScope ps(c, 1, s, ncol);
    const size_t total = (size_t)ncol * c->nz;
    const int blocks = (int)std::min<size_t>((total + 255) / 256, (size_t)c->nsm * 16);
    k_opac<<<blocks, 256, 0, s>>>(c->d_params, c->d_consts, ncol, d_mout, c->d_chem, c->d_slab, list, nlist);
  }
  FZ_CK(cudaGetLastError());
  const int threads = (c->numw + 31) & ~31;
  const size_t sms = (size_t)c->nz * c->sw * sizeof(float);
  {
    ProfScope ps(c, 2, s, ncol);
    // listed: a grid of 32 CTAs per SM walks the list
    const int grid = list ? std::min(ncol, c->nsm * 32) : ncol;
    k_synth<<<grid, threads, sms, s>>>(c->d_params, c->d_lam, c->d_gain, ncol, c->d_slab, d_syn, d_mout, d_status,
                                       list, nlist);
  }
  FZ_CK(cudaGetLastError());
  return launch_lsf<double>(c, d_syn, (long long)ncol * 4, 4, s, list, nlist);
}

size_t rf_smem(const fz_ctx* c) {
  const int threads = (c->numw + 31) & ~31;
  return ((size_t)rf_sums_off(c->nz, rf_w(c->nreg, c->nlu), c->rf.np, threads) + (size_t)24 * threads) *
         sizeof(float);
}

// the same for the FULL variant (no coefficient table or accumulators)
size_t rf_smem_full(const fz_ctx* c) {
  const int threads = (c->numw + 31) & ~31;
  return ((size_t)rf_sums_off(c->nz, rf_w(c->nreg, c->nlu), 0, threads) + (size_t)24 * threads) * sizeof(float);
}

// The response-function kernels run one thread per wavelength in blocks of
// at most 512: NUMW <= 512, and their shared memory within the 227 KB a
// block may have (the slab alone when the node Jacobian is contracted from
// the full response functions).
int rf_check(const fz_ctx* c) {
  if (((c->numw + 31) & ~31) > 512) return FZ_ERR_LIMIT;
  if ((c->rf_full ? rf_smem_full(c) : rf_smem(c)) > 227 * 1024) return FZ_ERR_LIMIT;
  return 0;
}

int ensure_rf_scratch(fz_ctx* c, int ncol) {
  int rc = ensure_scratch(c, ncol);
  if (rc) return rc;
  // the node kernels' shared memory above the default 48 KB (set here, before
  // any stream capture of the inversion's iteration)
  const int swr = rf_w(c->nreg, c->nlu);
  if (c->rf_full) {
    // the node Jacobian through the response functions at every height:
    // their scratch and the operators of k_rf_prop for ncol columns
    const size_t nrf = (size_t)ncol * NSLOT * c->nz * 4 * c->numw;
    if (nrf > c->rfbig_len) {
      cudaFree(c->d_rfbig);
      c->d_rfbig = nullptr;
      c->rfbig_len = 0;
      FZ_CK(cudaMalloc(&c->d_rfbig, nrf * sizeof(float)));
      c->rfbig_len = nrf;
    }
    const size_t nop = (size_t)ncol * c->nz * 16 * c->numw;
    if (nop > c->oscr_len) {
      cudaFree(c->d_oscr);
      c->d_oscr = nullptr;
      c->oscr_len = 0;
      FZ_CK(cudaMalloc(&c->d_oscr, nop * sizeof(float)));
      c->oscr_len = nop;
    }
    const size_t fsm = rf_smem_full(c);
    FZ_CK((set_synth_rf_attr<true, true>(cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm)));
    FZ_CK((set_synth_rf_attr<false, true>(cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm)));
  } else {
    const size_t sms = rf_smem(c);
    if (sms > 48 * 1024) {
      FZ_CK((set_synth_rf_attr<true, false>(cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sms)));
      FZ_CK((set_synth_rf_attr<false, false>(cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sms)));
    }
  }
  if ((size_t)ncol > c->rf_cols) {
    cudaFree(c->d_rfslab);
    cudaFree(c->d_chemd);
    c->d_rfslab = nullptr;
    c->d_chemd = nullptr;
    c->rf_cols = 0;
    FZ_CK(cudaMalloc(&c->d_rfslab, (size_t)ncol * c->nz * swr * sizeof(float)));
    FZ_CK(cudaMalloc(&c->d_chemd, (size_t)ncol * c->nz * sizeof(double4)));
    c->rf_cols = ncol;
  }
  return 0;
}

// The chemistry and opacity-derivative launches of the RF path with an
// explicit launch shape (the autotuner's candidates; c->tune otherwise).
void launch_chain(fz_ctx* c, int ncol, const float* d_model, float* d_mout, int* d_status, int hydrostatic, int wpb,
                  cudaStream_t s, int lanes = -1) {
  launch_k_chain(c, ncol, d_model, d_mout, d_status, hydrostatic, wpb, lanes >= 0 ? lanes : c->tune.chain_lanes, s);
}

// list / nlist (device): only the columns list[0 .. *nlist) of the first ncol
// (ncol bounds the grid); null: columns 0 .. ncol.
void launch_chemder(fz_ctx* c, int ncol, const float* d_mout, int bpsm, cudaStream_t s, const int* list = nullptr,
                    const int* nlist = nullptr) {
  const size_t cells = (size_t)ncol * c->nz;
  size_t blocks = (cells + 3) / 4;
  if (bpsm > 0) blocks = std::min<size_t>(blocks, (size_t)c->nsm * bpsm);
  k_chemder<<<(int)blocks, 128, 0, s>>>(c->d_params, c->d_consts, c->d_pf, c->d_pfd, ncol, d_mout, c->d_chem,
                                        c->d_chemd, list, nlist);
}

void launch_opac_rf(fz_ctx* c, int ncol, const float* d_mout, int threads, cudaStream_t s, const int* list = nullptr,
                    const int* nlist = nullptr) {
  const size_t cells = (size_t)ncol * c->nz;
  const int b2 = (int)std::min<size_t>((cells + threads - 1) / threads, (size_t)c->nsm * (4096 / threads));
  k_opac_rf<<<b2, threads, 0, s>>>(c->d_params, c->d_consts, ncol, d_mout, c->d_chem, c->d_chemd, c->d_rfslab, list,
                                   nlist);
}

// The response-function stage of the node path (chemistry derivatives,
// opacity derivatives, RF synthesis + node Jacobian) on columns whose
// chemistry k_chain has already left in the context's scratch.
int launch_rf_stage_full(fz_ctx* c, int ncol, int hydrostatic, double* d_syn, float* d_jac, float* d_mout,
                         int* d_status, cudaStream_t s, const int* list, const int* nlist);

int launch_rf_stage(fz_ctx* c, int ncol, int hydrostatic, double* d_syn, float* d_jac, float* d_mout, int* d_status,
                    cudaStream_t s, const int* list = nullptr, const int* nlist = nullptr) {
  if (c->rf_full) return launch_rf_stage_full(c, ncol, hydrostatic, d_syn, d_jac, d_mout, d_status, s, list, nlist);
  {
    ProfScope ps(c, 10, s, list ? 0 : ncol);
    launch_chemder(c, ncol, d_mout, c->tune.chemder_bpsm, s, list, nlist);
  }
  FZ_CK(cudaGetLastError());
  {
    ProfScope ps(c, 3, s, list ? 0 : ncol);
    launch_opac_rf(c, ncol, d_mout, c->tune.opacrf_threads, s, list, nlist);
  }
  FZ_CK(cudaGetLastError());
  const int threads = (c->numw + 31) & ~31;
  const size_t sms = rf_smem(c);
  {
    ProfScope ps(c, 4, s, list ? 0 : ncol);
    if (hydrostatic)
      launch_synth_rf<true, false>(has_blends(c), ncol, threads, sms, s, c->d_params, c->d_rf, c->d_lam, c->d_gain, ncol,
                                                         c->d_rfslab, c->d_coef, d_syn, d_jac, nullptr, d_mout,
                                                         d_status, list, nlist);
    else
      launch_synth_rf<false, false>(has_blends(c), ncol, threads, sms, s, c->d_params, c->d_rf, c->d_lam, c->d_gain, ncol,
                                                          c->d_rfslab, c->d_coef, d_syn, d_jac, nullptr, d_mout,
                                                          d_status, list, nlist);
  }
  FZ_CK(cudaGetLastError());
  if (c->lsf.on) {
    FZ_CK_RC(launch_lsf<double>(c, d_syn, (long long)ncol * 4, 4, s, list, nlist));
    FZ_CK_RC(launch_lsf<float>(c, d_jac, (long long)ncol * 4 * c->rf.np, 4 * c->rf.np, s, list, nlist));
  }
  return 0;
}

// The RF stage of node layouts too large for the forward accumulation: the
// response functions at every height of the columns (FULL synthesis,
// k_rf_prop with GAIN) into the context's scratch, contracted by the hat
// table into the node Jacobian (NFREQ, NP) per column of d_jac.  Scratch and
// kernel attributes come from ensure_rf_scratch (before any capture).
int launch_rf_stage_full(fz_ctx* c, int ncol, int hydrostatic, double* d_syn, float* d_jac, float* d_mout,
                         int* d_status, cudaStream_t s, const int* list, const int* nlist) {
  if (!c->d_rfbig || c->rfbig_len < (size_t)ncol * NSLOT * c->nz * 4 * c->numw) return FZ_ERR_STATE;
  {
    ProfScope ps(c, 10, s, list ? 0 : ncol);
    launch_chemder(c, ncol, d_mout, c->tune.chemder_bpsm, s, list, nlist);
  }
  FZ_CK(cudaGetLastError());
  {
    ProfScope ps(c, 3, s, list ? 0 : ncol);
    launch_opac_rf(c, ncol, d_mout, c->tune.opacrf_threads, s, list, nlist);
  }
  FZ_CK(cudaGetLastError());
  const int threads = (c->numw + 31) & ~31;
  const size_t sms = rf_smem_full(c);
  {
    ProfScope ps(c, 4, s, list ? 0 : ncol);
    if (hydrostatic)
      launch_synth_rf<true, true>(has_blends(c), ncol, threads, sms, s, c->d_params, c->d_rf, c->d_lam, c->d_gain,
                                  ncol, c->d_rfslab, nullptr, d_syn, c->d_rfbig, c->d_oscr, d_mout, d_status, list,
                                  nlist);
    else
      launch_synth_rf<false, true>(has_blends(c), ncol, threads, sms, s, c->d_params, c->d_rf, c->d_lam, c->d_gain,
                                   ncol, c->d_rfslab, nullptr, d_syn, c->d_rfbig, c->d_oscr, d_mout, d_status, list,
                                   nlist);
  }
  FZ_CK(cudaGetLastError());
  {
    ProfScope ps(c, 11, s, list ? 0 : ncol);
    k_rf_prop<<<ncol, threads, c->nz * sizeof(int), s>>>(c->nz, c->numw, c->d_gain, c->d_oscr, c->d_rfbig, list,
                                                         nlist);
  }
  FZ_CK(cudaGetLastError());
  const int nf = 4 * c->numw;
  k_rf_contract<<<dim3((nf + 255) / 256, c->rf.np, ncol), 256, 0, s>>>(c->nz, nf, c->rf, c->d_coef, c->d_rfbig,
                                                                       d_jac, list, nlist);
  FZ_CK(cudaGetLastError());
  if (c->lsf.on) {
    FZ_CK_RC(launch_lsf<double>(c, d_syn, (long long)ncol * 4, 4, s, list, nlist));
    FZ_CK_RC(launch_lsf<float>(c, d_jac, (long long)ncol * 4 * c->rf.np, 4 * c->rf.np, s, list, nlist));
  }
  return 0;
}

// full = false: node Jacobian (NFREQ, NP) per column with the layout of
// fz_rf_nodes; full = true: response functions at every height
// (NFREQ, 6 NZ) per column.
int launch_forward_rf(fz_ctx* c, int ncol, const float* d_model, int hydrostatic, double* d_syn, float* d_jac,
                      float* d_mout, int* d_status, cudaStream_t s, bool full = false) {
  if (hydrostatic < 0 || hydrostatic > 1) return FZ_ERR_ARG;   // RFs: HE from the top only
  if (!full && (c->rf.np <= 0 || !c->d_coef)) return FZ_ERR_STATE;
  if (int rc = rf_check(c)) return rc;
  int rc = ensure_rf_scratch(c, ncol);
  if (rc) return rc;
  const int swr = rf_w(c->nreg, c->nlu);
  if (d_status) FZ_CK(cudaMemsetAsync(d_status, 0, ncol * sizeof(int), s));
  launch_chain(c, ncol, d_model, d_mout, d_status, hydrostatic, c->tune.chain_warps, s);
  FZ_CK(cudaGetLastError());
  if (!full) return launch_rf_stage(c, ncol, hydrostatic, d_syn, d_jac, d_mout, d_status, s);
  {
    ProfScope ps(c, 10, s, ncol);
    launch_chemder(c, ncol, d_mout, c->tune.chemder_bpsm, s);
  }
  FZ_CK(cudaGetLastError());
  {
    ProfScope ps(c, 3, s, ncol);
    launch_opac_rf(c, ncol, d_mout, c->tune.opacrf_threads, s);
  }
  FZ_CK(cudaGetLastError());
  const int threads = (c->numw + 31) & ~31;
  {
    const size_t need = (size_t)ncol * c->nz * 16 * c->numw;
    if (need > c->oscr_len) {
      cudaFree(c->d_oscr);
      c->d_oscr = nullptr;
      c->oscr_len = 0;
      FZ_CK(cudaMalloc(&c->d_oscr, need * sizeof(float)));
      c->oscr_len = need;
    }
    const size_t sms = rf_smem_full(c);
    FZ_CK((set_synth_rf_attr<true, true>(cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sms)));
    FZ_CK((set_synth_rf_attr<false, true>(cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sms)));
    {
      ProfScope ps(c, 4, s, ncol);
      if (hydrostatic)
        launch_synth_rf<true, true>(has_blends(c), ncol, threads, sms, s, c->d_params, c->d_rf, c->d_lam, c->d_gain, ncol,
                                                          c->d_rfslab, nullptr, d_syn, d_jac, c->d_oscr, d_mout,
                                                          d_status, nullptr, nullptr);
      else
        launch_synth_rf<false, true>(has_blends(c), ncol, threads, sms, s, c->d_params, c->d_rf, c->d_lam, c->d_gain, ncol,
                                                           c->d_rfslab, nullptr, d_syn, d_jac, c->d_oscr, d_mout,
                                                           d_status, nullptr, nullptr);
    }
    FZ_CK(cudaGetLastError());
    {
      ProfScope ps(c, 11, s, ncol);
      k_rf_prop<<<ncol, threads, c->nz * sizeof(int), s>>>(c->nz, c->numw, c->d_gain, c->d_oscr, d_jac);
    }
    FZ_CK(cudaGetLastError());
    if (c->lsf.on) {
      FZ_CK_RC(launch_lsf<double>(c, d_syn, (long long)ncol * 4, 4, s));
      FZ_CK_RC(launch_lsf<float>(c, d_jac, (long long)ncol * 24 * c->nz, 24 * c->nz, s));
    }
    return 0;
  }
}

void lm_free_pool(LMSlots& L) {
  cudaFree(L.pix);
  cudaFree(L.skip);
  cudaFree(L.restarted);
  cudaFree(L.iter);
  cudaFree(L.st);
  cudaFree(L.mcur);
  cudaFree(L.mbest);
  cudaFree(L.syn);
  cudaFree(L.synb);
  cudaFree(L.jacb);
  cudaFree(L.need_rf);
  cudaFree(L.rf_list);
  cudaFree(L.pen);
  cudaFree(L.obs);
  cudaFree(L.diff);
  cudaFree(L.H);
  cudaFree(L.g);
  cudaFree(L.delta);
  cudaFree(L.status);
  L = LMSlots{};
}

void lm_free(fz_ctx* c) {
  lm_free_pool(c->lm);
  lm_free_pool(c->lm2);
  cudaFree(c->d_dest);
  c->d_dest = nullptr;
  cudaFree(c->d_act);
  c->d_act = nullptr;
  c->lm_cap = 0;
}

int lm_alloc_pool(LMSlots& L, int S, int np, int nf, int nm) {
  L.S = S;
  FZ_CK(cudaMalloc(&L.pix, S * sizeof(int)));
  FZ_CK(cudaMalloc(&L.skip, S * sizeof(int)));
  FZ_CK(cudaMalloc(&L.restarted, S * sizeof(int)));
  FZ_CK(cudaMalloc(&L.iter, S * sizeof(int)));
  FZ_CK(cudaMalloc(&L.st, 5 * (size_t)S * sizeof(double)));
  FZ_CK(cudaMalloc(&L.mcur, (size_t)S * nm * sizeof(float)));
  FZ_CK(cudaMalloc(&L.mbest, (size_t)S * nm * sizeof(float)));
  FZ_CK(cudaMalloc(&L.syn, (size_t)S * nf * sizeof(double)));
  FZ_CK(cudaMalloc(&L.synb, (size_t)S * nf * sizeof(double)));
  FZ_CK(cudaMalloc(&L.jacb, (size_t)S * np * nf * sizeof(float)));
  FZ_CK(cudaMalloc(&L.need_rf, (size_t)S * sizeof(int)));
  FZ_CK(cudaMalloc(&L.pen, (size_t)S * np * sizeof(double)));
  FZ_CK(cudaMalloc(&L.rf_list, (size_t)S * sizeof(int)));
  FZ_CK(cudaMalloc(&L.obs, (size_t)S * nf * sizeof(double)));
  FZ_CK(cudaMalloc(&L.diff, (size_t)S * nf * sizeof(double)));
  FZ_CK(cudaMalloc(&L.H, (size_t)S * np * np * sizeof(double)));
  FZ_CK(cudaMalloc(&L.g, (size_t)S * np * sizeof(double)));
  FZ_CK(cudaMalloc(&L.delta, (size_t)S * np * sizeof(double)));
  FZ_CK(cudaMalloc(&L.status, (size_t)S * sizeof(int)));
  return 0;
}

// slot pools for S slots of the current node layout
int lm_alloc(fz_ctx* c, int S) {
  const int np = c->rf.np, nf = 4 * c->numw, nm = 13 * c->nz;
  if ((size_t)S <= c->lm_cap && c->lm.S == S && c->lm_np == np) return 0;
  lm_free(c);
  c->lm_np = np;
  int rc = lm_alloc_pool(c->lm, S, np, nf, nm);
  if (!rc) rc = lm_alloc_pool(c->lm2, S, np, nf, nm);
  if (!rc) rc = cuda_fail(cudaMalloc(&c->d_dest, S * sizeof(int)));
  if (!rc) rc = cuda_fail(cudaMalloc(&c->d_act, S * sizeof(int)));
  if (rc) {
    lm_free(c);
    return rc;
  }
  c->lm_cap = S;
  return 0;
}

// ISIGMAP of SET_WEIGHTS (src/get_dmodel.f90:2024-2047) with the WSTK
// normalisation of src/input_file.f90:1298-1303, all Stokes inverted.
std::vector<double> lm_weights(int numw, const float wstk[4], double isigma) {
  float ss = 0.0f;
  for (int i = 0; i < 4; ++i) ss += wstk[i] * wstk[i];
  const float minw = std::sqrt(ss) / std::sqrt(4.0f);
  std::vector<double> w(4 * (size_t)numw);
  for (int i = 0; i < 4; ++i) {
    const float wi = wstk[i] / minw;
    for (int l = 0; l < numw; ++l) w[(size_t)i * numw + l] = (double)(wi * wi) / (isigma * isigma);
  }
  return w;
}

int lm_conf(fz_ctx* c, int npix, const fz_lm_opts* o, LMConf& C) {
  if (c->rf.np <= 0) return FZ_ERR_STATE;
  if (c->rf.np > LM_MAXNP_BIG) return FZ_ERR_LIMIT;
  const bool big = c->rf.np > LM_MAXNP;   // per-node tables in device memory
  static const int kRef[NSLOT] = {1, 2, 4, 5, 6, 7};
  static const int kRow[9] = {0, 0, 1, 2, 5, 6, 7, 10, 1};   // model row of reference parameter 1..8
  std::memset(&C, 0, sizeof(C));
  C.np = c->rf.np;
  C.nfreq = 4 * c->numw;
  C.nz = c->nz;
  C.npix = npix;
  C.maxsteps = o && o->maxsteps > 0 ? o->maxsteps : 5;
  C.maxit = o && o->maxit > 0 ? o->maxit : 40;
  C.dchi2 = o ? o->dchi2 : 0.0;
  C.svdtol = o && o->svdtol > 0 ? o->svdtol : 1.0e-4;
  C.inu = (double)C.nfreq;
  C.fallback = o && o->fallback_model ? o->fallback : 0.0;
  C.fb_model = o ? o->fallback_model : nullptr;
  // fallback_steps > 0: at that STEPS count; < 0: at the first evaluation; 0: when the search ends
  C.fb_steps = o && o->fallback_steps > 0 ? o->fallback_steps : (o && o->fallback_steps < 0 ? 0 : (1 << 30));
  C.fb_free = o && o->fallback_free ? 1 : 0;
  C.solver = o && o->solver == 2 ? 2 : 1;
  C.node_exp = o && o->node_expansion == 2 ? 2 : 1;
  C.global_stop = o && o->global_stop ? 1 : 0;
  C.state_out = o ? o->state_out : nullptr;
  if (o && o->cycles_left < 0) return FZ_ERR_ARG;
  if (o && (o->solver < 0 || o->solver > 2 || o->node_expansion < 0 || o->node_expansion > 2)) return FZ_ERR_ARG;
  // GET_IT_PENALTIES operators (src/get_dmodel.f90:1103-1146): per free
  // parameter L = sqrt(PEN_ALP / IFREEP) D, D = diag(1/NJ) (type 0) or first
  // differences to the previous node (type 1); PEN_HSS = L^T L block diagonal
  if (o)
    for (int p = 0; p < 8; ++p)
      if (o->reg_alpha[p] < 0.0 || (o->reg_alpha[p] > 0.0 && o->reg_type[p] != 0 && o->reg_type[p] != 1))
        return FZ_ERR_ARG;
  const double norms[8] = {6000.0, 1.0e5, 1.0e-5, 1.0e3, 1.0e3, 1.0e3, 1.0e6, 6.0e2};
  // nodes in reference parameter order (the slot order of the Jacobian)
  for (int p = 0; p < NSLOT; ++p) {
    const int rp = kRef[p];
    C.nodes_ref[rp - 1] = c->rf.nj[p];
    for (int j = 0; !big && j < c->rf.nj[p]; ++j) {
      const int n = c->rf.n0[p] + j;
      C.row_of[n] = kRow[rp];
      C.par_of[n] = rp;
      C.norm[n] = norms[rp - 1];
    }
  }
  C.d_row = c->d_nrow;
  C.d_norm = c->d_nnorm;
  std::vector<double> hbig;
  if (big) hbig.assign((size_t)C.np * C.np, 0.0);
  if (o) {
    for (int p = 0; p < NSLOT; ++p) {
      const int rp = kRef[p], nj = c->rf.nj[p], j0 = c->rf.n0[p];
      const double alp = o->reg_alpha[rp - 1];
      if (nj <= 0 || alp <= 0.0) continue;
      C.reg = 1;
      const double a2 = alp / (double)C.np;   // ALP^2
      for (int k = 0; k < nj; ++k)
        for (int l = 0; l < nj; ++l) {
          double v = 0.0;   // (D^T D)(k, l)
          if (o->reg_type[rp - 1] == 0) {
            v = k == l ? 1.0 / ((double)nj * nj) : 0.0;
          } else {
            // D rows r >= 1: e_r - e_{r-1}
            for (int r = 1; r < nj; ++r) {
              const double dk = (k == r ? 1.0 : 0.0) - (k == r - 1 ? 1.0 : 0.0);
              const double dl = (l == r ? 1.0 : 0.0) - (l == r - 1 ? 1.0 : 0.0);
              v += dk * dl;
            }
          }
          if (big)
            hbig[(size_t)(j0 + k) * C.np + (j0 + l)] = a2 * v;
          else
            C.reg_hss[(j0 + k) * C.np + (j0 + l)] = a2 * v;
        }
    }
  }
  if (big && C.reg) {
    // PEN_HSS of a large layout in device memory, uploaded when it changes
    // (after the device has finished with the previous one)
    if (hbig != c->nhss_host) {
      FZ_CK(cudaDeviceSynchronize());
      cudaFree(c->d_nhss);
      c->d_nhss = nullptr;
      c->nhss_host.clear();
      FZ_CK(cudaMalloc(&c->d_nhss, hbig.size() * sizeof(double)));
      FZ_CK(cudaMemcpy(c->d_nhss, hbig.data(), hbig.size() * sizeof(double), cudaMemcpyHostToDevice));
      c->nhss_host = hbig;
    }
    C.d_hss = c->d_nhss;
  }
  return 0;
}

// GET_INT_COEFS with GET_POSITIONS (src/get_dmodel.f90:452-466, 563-644):
// hat functions on equally spaced node positions, coef(height, node).
bool int_coefs(int nz, int nj, std::vector<double>& coef) {
  coef.assign((size_t)nz * nj, 0.0);
  if (nj == 1) {
    for (int i = 0; i < nz; ++i) coef[i] = 1.0;
  } else if (nj < nz) {
    std::vector<double> pos(nj);
    const double step = (double)(nz - 1) / (double)(nj - 1);
    for (int i = 1; i <= nj; ++i) pos[i - 1] = ((double)i - 1.0) * step + 1.0;
    for (int j = 1; j <= nj; ++j) {
      const double ji = pos[std::max(j - 1, 1) - 1], jf = pos[std::min(j + 1, nj) - 1], jm = pos[j - 1];
      for (int i = 1; i <= nz; ++i) {
        const double di = (double)i;
        if (di < ji || di > jf) continue;
        double v;
        if (di == jm) v = 1.0;
        else if (di < jm) v = 1.0 / (jm - ji) * (di - ji);
        else v = 1.0 / (jf - jm) * (jf - di);
        coef[(size_t)(j - 1) * nz + (i - 1)] = v;
      }
    }
  } else if (nj == nz) {
    for (int i = 0; i < nz; ++i) coef[(size_t)i * nz + i] = 1.0;
  } else {
    return false;
  }
  return true;
}

// ------------------------------------------------------------- log tau5
// The GETTAU mode (MODE t, src/invert3d.f90:159-178 with MSYNTHESIS off):
// log tau5 of every column from the opacity slab k_opac leaves, the
// integration of src/forward.f90:1000-1006 (REAL*4 accumulation from the
// top, as k_synth does), without the Stokes synthesis.
// Grid-stride FP64 -> FP32 rounding (a REAL*8 Jacobian into the FP32
// operand of the split-bf16 normal equations).
__global__ void k_f64_to_f32(size_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// Warm-start models, one CTA per pixel: the network's outputs y (node order
// of the layout, standardised) become node values v = y tsd + tmu, and each
// free parameter's row of the base model (13, nz) is moved by
// EXPAND(v - CONTRACT(base)) -- the way the inversion perturbs a model
// (CONTRACT_VECTOR / EXPAND_VECTOR, src/get_dmodel.f90:839-880); the other
// rows are the base model's.  coef: the (nz, np) hat table in FP32.
// CONTRACT(base) of the one base model every pixel shares: node j's hat
// average of its parameter's row (one thread per node, once per call).
__global__ void k_ws_contract(int nz, RFConf R, const float* __restrict__ coef, const float* __restrict__ base,
                              float* __restrict__ cb) {
  static const int kRow[NSLOT] = {0, 1, 5, 6, 7, 10};   // model rows of T, Pg, Bx, By, Bz, v_z
  const int np = R.np;
  for (int j = threadIdx.x; j < np; j += blockDim.x) {
    int p = 0;
    while (p < NSLOT - 1 && j >= R.n0[p] + R.nj[p]) ++p;
    const float* b = base + kRow[p] * nz;
    float a = 0.0f, cs = 0.0f;
    for (int k = 0; k < nz; ++k) cs += coef[(size_t)k * np + j];
    for (int k = 0; k < nz; ++k) a += b[k] * (coef[(size_t)k * np + j] / cs);
    cb[j] = a;
  }
}

__global__ void __launch_bounds__(128) k_ws_expand(int npix, int nz, RFConf R, const float* __restrict__ coef,
                                                   const float* __restrict__ y, const float* __restrict__ tmu,
                                                   const float* __restrict__ tsd, const float* __restrict__ base,
                                                   const float* __restrict__ cb, float* __restrict__ out) {
  extern __shared__ float wsv[];   // np node offsets v - CONTRACT(base)
  static const int kRow[NSLOT] = {0, 1, 5, 6, 7, 10};   // model rows of T, Pg, Bx, By, Bz, v_z
  const int pix = blockIdx.x;
  const int np = R.np;
  float* m = out + (size_t)pix * 13 * nz;
  for (int i = threadIdx.x; i < 13 * nz; i += blockDim.x) m[i] = base[i];
  for (int j = threadIdx.x; j < np; j += blockDim.x) wsv[j] = fmaf(y[(size_t)pix * np + j], tsd[j], tmu[j]) - cb[j];
  __syncthreads();
  for (int p = 0; p < NSLOT; ++p) {
    if (R.nj[p] == 0) continue;
    float* row = m + kRow[p] * nz;
    const float* b = base + kRow[p] * nz;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
      float d = 0.0f;
      for (int j = R.n0[p]; j < R.n0[p] + R.nj[p]; ++j) d = fmaf(wsv[j], coef[(size_t)k * np + j], d);
      row[k] = b[k] + d;
    }
  }
}

// The formal solution alone on given absorption matrices (SET_BOUNDARY +
// OLD_ANALYTICAL_SOLVER): one thread per (column, wavelength), the height
// recursion of the synthesis kernel with the layer optical depths
// eta * dz (dz from the reference's rule: z_{k+1} - z_k, the top height's
// backward difference).  eta (nw, 7, nz, ncol), src (nw, nz, ncol), bnd
// (nz, ncol) or null, out (4, nw, ncol).
__global__ void k_rte(int ncol, int nz, int nw, const float* __restrict__ eta, const float* __restrict__ src,
                      const double* __restrict__ zz, const int* __restrict__ bnd, double* __restrict__ out) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)ncol * nw) return;
  const int col = (int)(idx / nw), l = (int)(idx % nw);
  float I0 = 0.f, I1 = 0.f, I2 = 0.f, I3 = 0.f;
  for (int k = 0; k < nz; ++k) {
    const float S = src[((size_t)col * nz + k) * nw + l];
    if (k == 0 || (bnd && bnd[(size_t)col * nz + k])) {
      I0 = S;
      I1 = I2 = I3 = 0.f;
      continue;
    }
    const double dz = 1e5 * fabs(k == nz - 1 ? zz[k] - zz[k - 1] : zz[k + 1] - zz[k]);
    const float* e = eta + ((size_t)col * nz + k) * 7 * nw + l;
    float t[7];
    bool fin = true;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
      t[i] = (float)((double)e[(size_t)i * nw] * dz);
      fin = fin && isfinite(t[i]);
    }
    float O[16], om0 = 0.0f;
    if (!fin) {
#pragma unroll
      for (int i = 0; i < 16; ++i) O[i] = (i % 5 == 0) ? 1.f : 0.f;
    } else {
      evol_f32(t[0], t[1], t[2], t[3], t[4], t[5], t[6], O, om0);
    }
    rte_step(O, om0, S, I0, I1, I2, I3);
  }
  double* o = out + ((size_t)col * nw + l) * 4;
  o[0] = I0;
  o[1] = I1;
  o[2] = I2;
  o[3] = I3;
}

// VOIGT on arrays: the FP32 Voigt/Faraday-Voigt pair of the synthesis kernels.
__global__ void k_voigt(int n, const float* __restrict__ a, const float* __restrict__ v, float* __restrict__ h,
                        float* __restrict__ f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float hh, ff;
  voigt_f32(a[i], v[i], hh, ff);
  h[i] = hh;
  f[i] = ff;
}

__global__ void k_tau5(int ncol, int nz, int sw, const float* __restrict__ slab, float* __restrict__ mout) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const float* sm = slab + (size_t)col * nz * sw;
  float* mo = mout + (size_t)col * 13 * nz;
  float tau = 1e-9f;
  mo[11 * nz + nz - 1] = log10f(tau);
  for (int k = nz - 2; k >= 0; --k) {
    const float a = (sm[k * sw + 2] * sm[k * sw + 3] + sm[(k + 1) * sw + 2] * sm[(k + 1) * sw + 3]) / 2.0f;
    const double b = ((double)mo[12 * nz + k + 1] - (double)mo[12 * nz + k]) * 1000.0 * 100.0;
    tau = (float)((double)tau + (double)a * b);
    mo[11 * nz + k] = log10f(tau);
  }
}

// ------------------------------------------------------------ SMOOTHING_B
// The 1-2-1 smoothing of the free parameters' cubes at the start of every
// cycle (SMOOTHING_B, src/model_spatial_extension.f90:351-491, called from
// INITIALIZE_CYCLE, src/invert3d.f90:228-325): in FP64, along x (pixels
// iy + NY ix), then y, then z, each pass on the previous pass's whole array
// (array assignment), the first and last index of a direction kept, a
// direction of 4 or fewer points left alone; the result rounded to REAL*4.
// Buffers: (nrow, npix, nz) doubles.
__global__ void k_smooth_load(int npix, int nz, int nrow, const int* __restrict__ rows, const float* __restrict__ m,
                              double* __restrict__ a) {
  const size_t total = (size_t)nrow * npix * nz;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % nz);
    const size_t pr = i / nz;
    const int pix = (int)(pr % npix), r = (int)(pr / npix);
    a[i] = (double)m[((size_t)pix * 13 + rows[r]) * nz + k];
  }
}

// dir 0: x (stride NY pixels), 1: y (stride 1 pixel), 2: z; the last pass
// writes REAL*4 into the model rows.  A shard of the field holds columns
// x0g .. of an nxg-column field (the edge and 4-point rules are the
// field's), its array extended by the neighbours' halo columns.
__global__ void k_smooth_pass(int nx, int ny, int nz, int nrow, int dir, const int* __restrict__ rows,
                              const double* __restrict__ a, double* __restrict__ b, float* __restrict__ m,
                              int x0g, int nxg) {
  const int npix = nx * ny;
  const size_t total = (size_t)nrow * npix * nz;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % nz);
    const size_t pr = i / nz;
    const int pix = (int)(pr % npix), r = (int)(pr / npix);
    const int iy = pix % ny, ix = pix / ny;
    double v = a[i];
    const int gx = ix + x0g;   // the field's column
    if (dir == 0 && nxg > 4 && gx > 0 && gx < nxg - 1 && ix > 0 && ix < nx - 1)
      v = __dadd_rn(__dadd_rn(a[i + (size_t)ny * nz], a[i - (size_t)ny * nz]), __dmul_rn(v, 2.0)) / 4.0;
    else if (dir == 1 && ny > 4 && iy > 0 && iy < ny - 1)
      v = __dadd_rn(__dadd_rn(a[i + nz], a[i - nz]), __dmul_rn(v, 2.0)) / 4.0;
    else if (dir == 2 && nz > 4 && k > 0 && k < nz - 1)
      v = __dadd_rn(__dadd_rn(a[i + 1], a[i - 1]), __dmul_rn(v, 2.0)) / 4.0;
    if (m)
      m[((size_t)pix * 13 + rows[r]) * nz + k] = (float)v;
    else
      b[i] = v;
  }
}

// ------------------------------------------------------------- SET_TAU
// The assists of SET_TAU (src/invert3d.f90:492-727): field-wide template
// vectors from the summed Stokes I of the first spectral region, per-pixel
// projections, field maxima, then per-pixel rewrites of B, v_z, T and Pg.
// Pixels iy + NY ix; obs (npix, 4, numw) REAL*8 (OBS3D).

// Partial sums of Stokes I over y for every x (SUM(SUM(OBS3D(..),DIM=2),DIM=2)
// takes the y sum first): one thread per (x, wavelength of region 1).
__global__ void k_tau_ysum(int nx, int ny, int numw, int n1, const double* __restrict__ obs,
                           double* __restrict__ part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx * n1) return;
  const int ix = i / n1, j = i % n1;
  double t = 0.0;
  for (int iy = 0; iy < ny; ++iy) t += obs[((size_t)ix * ny + iy) * 4 * numw + j];
  part[i] = t;
}

// then over x, in order: one thread per wavelength
__global__ void k_tau_xsum(int nx, int n1, const double* __restrict__ part, double* __restrict__ tot) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n1) return;
  double t = 0.0;
  for (int ix = 0; ix < nx; ++ix) t += part[(size_t)ix * n1 + j];
  tot[j] = t;
}

// One warp per pixel: the projections of region 1 (vec = the three template
// vectors, 3 x n1): proj[p] = {V.v2, Q.v3, U.v3, I.v2, I.v1, mean I}.
__global__ void k_tau_proj(int npix, int numw, int n1, const double* __restrict__ obs, const double* __restrict__ vec,
                           double* __restrict__ proj) {
  const int lane = threadIdx.x & 31;
  const size_t p = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (p >= (size_t)npix) return;
  const double* o = obs + p * 4 * numw;
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int j = lane; j < n1; j += 32) {
    const double I = o[j], Q = o[numw + j], U = o[2 * numw + j], V = o[3 * numw + j];
    a[0] += V * vec[n1 + j];
    a[1] += Q * vec[2 * n1 + j];
    a[2] += U * vec[2 * n1 + j];
    a[3] += I * vec[n1 + j];
    a[4] += I * vec[j];
    a[5] += I;
  }
#pragma unroll
  for (int q = 0; q < 6; ++q)
    for (int off = 16; off > 0; off >>= 1) a[q] += __shfl_xor_sync(0xffffffffu, a[q], off);
  if (lane == 0) {
    for (int q = 0; q < 5; ++q) proj[p * 6 + q] = a[q];
    proj[p * 6 + 5] = a[5] / (double)n1;   // SUM(DBLE(I)) / DBLE(n)
  }
}

// Field maxima |V.v2|, sqrt((Q.v3)^2 + (U.v3)^2), |I.v2 - I.v1 KOL| as
// order-independent atomic maxima of non-negative doubles (bit patterns
// order like the values); mx zeroed by the caller.
__global__ void k_tau_max(int npix, double kol, const double* __restrict__ proj, unsigned long long* __restrict__ mx) {
  double m0 = 0.0, m1 = 0.0, m2 = 0.0;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < (size_t)npix; p += (size_t)gridDim.x * blockDim.x) {
    const double* q = proj + p * 6;
    m0 = fmax(m0, fabs(q[0]));
    m1 = fmax(m1, sqrt(q[1] * q[1] + q[2] * q[2]));
    m2 = fmax(m2, fabs(q[3] - q[4] * kol));
  }
  for (int off = 16; off > 0; off >>= 1) {
    m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, off));
    m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, off));
    m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(mx + 0, (unsigned long long)__double_as_longlong(m0));
    atomicMax(mx + 1, (unsigned long long)__double_as_longlong(m1));
    atomicMax(mx + 2, (unsigned long long)__double_as_longlong(m2));
  }
}

struct TauConf {
  int assist;     // 1 T, 2 Pg, 4 B, 8 v_z
  int nz, itz;    // ITZ - 1 = CEILING(NZ/3) - 1
  double kol, lk_hc;
};

// One warp per pixel: the assists in the reference's order B, v_z, T, Pg,
// with its REAL*4 / REAL*8 mixing (invert3d.f90:563-570, :621-625,
// :640-652, :666-671).
__global__ void k_tau_apply(TauConf C, int npix, const double* __restrict__ proj,
                            const unsigned long long* __restrict__ mx, float* __restrict__ models) {
  const int lane = threadIdx.x & 31;
  const size_t p = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (p >= (size_t)npix) return;
  const int nz = C.nz;
  float* m = models + p * 13 * nz;
  const double* q = proj + p * 6;
  if (C.assist & 4) {
    const double t3 = q[0] / __longlong_as_double((long long)mx[0]);
    const double t4 = sqrt(q[1] * q[1] + q[2] * q[2]) / __longlong_as_double((long long)mx[1]);
    const double atn2 = atan2(q[2], q[1]) / 2.0;
    const float bx = (float)((double)(-(float)sin(atn2) * 1000.0f) * t4);
    const float by = (float)((double)((float)cos(atn2) * 1000.0f) * t4);
    const float bz = (float)t3 * (-1000.0f);
    for (int k = lane; k < nz; k += 32) {
      m[5 * nz + k] = bx;
      m[6 * nz + k] = by;
      m[7 * nz + k] = bz;
    }
  }
  if (C.assist & 8) {
    const double d = (q[3] - q[4] * C.kol) / __longlong_as_double((long long)mx[2]);
    const float vz = (float)d * (-2.0e5f);
    for (int k = lane; k < nz; k += 32) m[10 * nz + k] = vz;
  }
  __syncwarp();
  if (C.assist & 1) {
    const double imean = q[5];
    const double tb = 1.0 / (C.lk_hc * log(1.0 + 1.0 / imean * (exp(1.0 / 6.39e3 / C.lk_hc) - 1.0)));
    const double sh = tb - (double)m[C.itz];
    __syncwarp();
    for (int k = lane; k < nz; k += 32) m[k] = (float)((double)m[k] + sh);
  }
  __syncwarp();
  if (C.assist & 2) {
    const float p0 = m[nz + C.itz];
    __syncwarp();
    for (int k = lane; k < nz; k += 32) m[nz + k] = m[nz + k] * 1.333e5f / p0;
  }
  if (C.assist & 3)
    for (int k = lane; k < nz; k += 32) m[11 * nz + k] = k == C.itz ? 0.0f : 1.0f;
}

// ------------------------------------------------------------ v3 layouts
// Cube of the v3 model file feeding each MODEL row (-1: vx, vy, zero; the
// file has no cube for them): JOIN_MODEL2 (src/forward.f90:363-405) over the
// cubes of READ_MODEL_3D (src/misc.f90:459-491).
__constant__ int c_v3_cube_of_row[13] = {0, 1, 2, 7, 8, 3, 4, 5, -1, -1, 6, 9, 12};
// MODEL row written into each of the first ten cubes (WRITE_MODEL3D_V3)
__constant__ int c_v3_row_of_cube[10] = {0, 1, 2, 5, 6, 7, 10, 3, 4, 11};

// One warp per (pixel, model row) or (cube, pixel): both sides hold the
// row as a contiguous run of nz values, moved as float4 when nz is a
// multiple of 4 and both bases are 16-byte aligned (vec), else as floats.
__device__ __forceinline__ void warp_copy(const float* __restrict__ src, float* __restrict__ dst, int nz, bool vec,
                                          int lane) {
  if (vec) {
    const float4* s4 = reinterpret_cast<const float4*>(src);
    float4* d4 = reinterpret_cast<float4*>(dst);
    for (int i = lane; i < (nz >> 2); i += 32) d4[i] = s4[i];
  } else {
    for (int i = lane; i < nz; i += 32) dst[i] = src[i];
  }
}

__device__ __forceinline__ void warp_fill(float v, float* __restrict__ dst, int nz, bool vec, int lane) {
  if (vec) {
    float4* d4 = reinterpret_cast<float4*>(dst);
    for (int i = lane; i < (nz >> 2); i += 32) d4[i] = make_float4(v, v, v, v);
  } else {
    for (int i = lane; i < nz; i += 32) dst[i] = v;
  }
}

__global__ void k_model_from_v3(int npix, int nz, bool vec, const float* __restrict__ cubes,
                                float* __restrict__ model) {
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  const size_t cube = (size_t)npix * nz, pairs = (size_t)npix * 13;
  for (size_t pr = (size_t)blockIdx.x * wpb + (threadIdx.x >> 5); pr < pairs; pr += (size_t)gridDim.x * wpb) {
    const int row = (int)(pr % 13);
    const size_t p = pr / 13;
    const int c = c_v3_cube_of_row[row];
    float* dst = model + pr * nz;
    if (c < 0)
      warp_fill(0.0f, dst, nz, vec, lane);
    else   // the z row: ZZ, the first pixel's z column
      warp_copy(c == 12 ? cubes + 12 * cube : cubes + (size_t)c * cube + p * nz, dst, nz, vec, lane);
  }
}

__global__ void k_model_to_v3(int ny, int npix, int nz, bool vec, const float* __restrict__ model,
                              const double* __restrict__ x, const double* __restrict__ y, float* __restrict__ cubes) {
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  const size_t pairs = (size_t)npix * 13;
  for (size_t cp = (size_t)blockIdx.x * wpb + (threadIdx.x >> 5); cp < pairs; cp += (size_t)gridDim.x * wpb) {
    const int c = (int)(cp / npix);
    const size_t p = cp % npix;
    float* dst = cubes + cp * nz;
    if (c == 10)
      warp_fill((float)x[p / ny], dst, nz, vec, lane);
    else if (c == 11)
      warp_fill((float)y[p % ny], dst, nz, vec, lane);
    else
      warp_copy(model + (p * 13 + (c < 10 ? c_v3_row_of_cube[c] : 12)) * nz, dst, nz, vec, lane);
  }
}

// STOKES(4,NW,npix) REAL*4 <-> OBS3D/RSYN1D(4*NW,npix) REAL*8 (Stokes-major
// blocks): one thread per (pixel, wavelength), its four Stokes values.
__global__ void k_obs_from_v3(int npix, int nw, const float* __restrict__ st, double* __restrict__ obs) {
  const size_t total = (size_t)npix * nw;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t p = i / nw;
    const int w = (int)(i % nw);
    const float* s = st + 4 * i;
    double* o = obs + p * 4 * nw + w;
#pragma unroll
    for (int q = 0; q < 4; ++q) o[(size_t)q * nw] = (double)s[q];
  }
}

__global__ void k_syn_to_v3(int npix, int nw, const double* __restrict__ syn, float* __restrict__ st) {
  const size_t total = (size_t)npix * nw;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t p = i / nw;
    const int w = (int)(i % nw);
    const double* s = syn + p * 4 * nw + w;
    float* o = st + 4 * i;
#pragma unroll
    for (int q = 0; q < 4; ++q) o[q] = (float)s[(size_t)q * nw];
  }
}

// The RF payload of WRITE_RFS3D_V3 from fz_forward_rf_full's output: one
// thread per (pixel, height, wavelength, Stokes) gathers the six parameters'
// responses (for a warp: four Stokes rows, 8 consecutive wavelengths each)
// and stores them as one run of six floats (a warp: 768 contiguous bytes).
__global__ void k_rf_to_v3(int npix, int nz, int nw, const float* __restrict__ rf, float* __restrict__ out) {
  const int nf = 4 * nw;
  const size_t total = (size_t)npix * nz * nf;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i % nf);   // w * 4 + s
    const size_t pk = i / nf;      // p * nz + k
    const size_t p = pk / nz;
    const int k = (int)(pk % nz);
    const int w = r >> 2, s = r & 3;
    const float* src = rf + (p * 6 * nz + k) * nf + s * nw + w;
    float v[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) v[q] = src[(size_t)q * nz * nf];
    float2* d = reinterpret_cast<float2*>(out + i * 6);
    d[0] = make_float2(v[0], v[1]);
    d[1] = make_float2(v[2], v[3]);
    d[2] = make_float2(v[4], v[5]);
  }
}

int grid_for(size_t n, int threads) {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return (int)std::max<size_t>(1, std::min<size_t>((n + threads - 1) / threads, (size_t)nsm * 16));
}

}  // namespace

extern "C" {

int fz_smooth_shard_device(fz_ctx* c, int nx, int ny, int x0, int nx_field, float* d_models, const int* params,
                           void* stream) {
  if (!c || nx <= 0 || ny <= 0 || !d_models || x0 < 0 || nx_field < x0 + nx) return FZ_ERR_ARG;
  // model row of reference parameter 1..8 (P0 smooths Pg, as the reference)
  static const int kRow[9] = {0, 0, 1, 2, 5, 6, 7, 10, 1};
  static const int kRef[NSLOT] = {1, 2, 4, 5, 6, 7};
  int rows[8], nrow = 0;
  for (int p = 1; p <= 8; ++p) {
    bool on;
    if (params) {
      on = params[p - 1] != 0;
    } else {
      on = false;
      for (int q = 0; q < NSLOT; ++q) on = on || (kRef[q] == p && c->rf.np > 0 && c->rf.nj[q] > 0);
    }
    if (on) rows[nrow++] = kRow[p];
  }
  if (nrow == 0) return 0;
  FZ_CK(cudaSetDevice(c->device));
  cudaStream_t s = (cudaStream_t)stream;
  const size_t npix = (size_t)nx * ny, n = (size_t)nrow * npix * c->nz;
  if (n > c->smooth_len) {
    FZ_CK(cudaStreamSynchronize(s));
    cudaFree(c->d_smooth);
    c->d_smooth = nullptr;
    c->smooth_len = 0;
    FZ_CK(cudaMalloc(&c->d_smooth, 2 * n * sizeof(double) + 8 * sizeof(int)));
    c->smooth_len = n;
  }
  double* a = c->d_smooth;
  double* b = a + n;
  int* d_rows = reinterpret_cast<int*>(b + n);
  FZ_CK(cudaMemcpyAsync(d_rows, rows, nrow * sizeof(int), cudaMemcpyHostToDevice, s));
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)c->nsm * 32);
  k_smooth_load<<<blocks, 256, 0, s>>>((int)npix, c->nz, nrow, d_rows, d_models, a);
  k_smooth_pass<<<blocks, 256, 0, s>>>(nx, ny, c->nz, nrow, 0, d_rows, a, b, nullptr, x0, nx_field);
  k_smooth_pass<<<blocks, 256, 0, s>>>(nx, ny, c->nz, nrow, 1, d_rows, b, a, nullptr, x0, nx_field);
  k_smooth_pass<<<blocks, 256, 0, s>>>(nx, ny, c->nz, nrow, 2, d_rows, a, nullptr, d_models, x0, nx_field);
  FZ_CK(cudaGetLastError());
  return 0;
}

int fz_smooth_device(fz_ctx* c, int nx, int ny, float* d_models, const int* params, void* stream) {
  return fz_smooth_shard_device(c, nx, ny, 0, nx, d_models, params, stream);
}

int fz_invert_cycles_device(fz_ctx* c, int nx, int ny, const double* d_obs, float* d_models, int ncycles,
                            const int* nodes, int hydrostatic, const fz_lm_opts* opts, double* d_chi2, int* d_iters,
                            int* d_status, void* stream) {
  if (!c || nx <= 0 || ny <= 0 || !d_obs || !d_models || ncycles <= 0 || !nodes || !d_chi2 || !d_iters)
    return FZ_ERR_ARG;
  if (hydrostatic < 0 || hydrostatic > 1) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  const int npix = nx * ny;
  const size_t nm = 13 * (size_t)c->nz;
  cudaStream_t s = (cudaStream_t)stream;
  float* d_best = nullptr;
  double* d_syn = nullptr;
  int rc = 0;
  do {
    if ((rc = cuda_fail(cudaMalloc(&d_best, (size_t)npix * nm * sizeof(float))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_syn, (size_t)npix * 4 * c->numw * sizeof(double))))) break;
    for (int cy = 0; cy < ncycles && !rc; ++cy) {
      // INITIALIZE_CYCLE: the cycle's node layout, SMOOTHING_B of the models
      if ((rc = cuda_fail(cudaStreamSynchronize(s)))) break;
      if ((rc = fz_rf_nodes(c, nodes + 8 * cy)) < 0) break;   // >= 0: the layout's NP
      rc = 0;
      // SET_TAU's assists when neither Pg nor P0 is free, every cycle or,
      // with PROGRESSIVE, the first only (invert3d.f90:505-520)
      const int assist = opts ? (opts->assist & 15) : 0;
      if (assist && nodes[8 * cy + 1] == 0 && nodes[8 * cy + 7] == 0 && (cy == 0 || !(opts->assist & 16)))
        if ((rc = fz_set_tau_device(c, nx, ny, d_obs, d_models, assist, hydrostatic, s))) break;
      if ((rc = fz_smooth_device(c, nx, ny, d_models, nullptr, s))) break;
      // the cycle's iterations, each pixel from a fresh LM state; the field
      // rule's threshold depends on the cycles still to come
      fz_lm_opts oc{};
      if (opts) oc = *opts;
      oc.cycles_left = ncycles - 1 - cy;
      if ((rc = fz_invert_device(c, npix, d_obs, d_models, nullptr, hydrostatic, opts ? &oc : nullptr, d_best, d_chi2,
                                 d_iters, nullptr, d_status, s)))
        break;
      // END_CYCLE: the best models through a plain synthesis (the derived
      // rows: Pg in hydrostatic mode, rho, Pe, mu, log tau5)
      if ((rc = launch_forward(c, npix, d_best, hydrostatic, d_syn, d_models, nullptr, s))) break;
    }
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(s));
  } while (false);
  cudaFree(d_best);
  cudaFree(d_syn);
  return rc;
}

int fz_model_from_v3_device(int nx, int ny, int nz, const float* d_cubes, float* d_model, void* stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || !d_cubes || !d_model) return FZ_ERR_ARG;
  const int npix = nx * ny;
  const bool vec = (nz & 3) == 0 && ((uintptr_t)d_cubes & 15) == 0 && ((uintptr_t)d_model & 15) == 0;
  k_model_from_v3<<<grid_for((size_t)npix * 13 * 32, 256), 256, 0, (cudaStream_t)stream>>>(npix, nz, vec, d_cubes,
                                                                                              d_model);
  return cuda_fail(cudaGetLastError());
}

int fz_model_to_v3_device(int nx, int ny, int nz, const float* d_model, const double* x, const double* y,
                          float* d_cubes, void* stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || !d_model || !x || !y || !d_cubes) return FZ_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  double* d_xy = nullptr;
  FZ_CK(cudaMalloc(&d_xy, (size_t)(nx + ny) * sizeof(double)));
  int rc = cuda_fail(cudaMemcpyAsync(d_xy, x, nx * sizeof(double), cudaMemcpyHostToDevice, s));
  if (!rc) rc = cuda_fail(cudaMemcpyAsync(d_xy + nx, y, ny * sizeof(double), cudaMemcpyHostToDevice, s));
  if (!rc) {
    const int npix = nx * ny;
    const bool vec = (nz & 3) == 0 && ((uintptr_t)d_model & 15) == 0 && ((uintptr_t)d_cubes & 15) == 0;
    k_model_to_v3<<<grid_for((size_t)npix * 13 * 32, 256), 256, 0, s>>>(ny, npix, nz, vec, d_model, d_xy,
                                                                         d_xy + nx, d_cubes);
    rc = cuda_fail(cudaGetLastError());
  }
  if (!rc) rc = cuda_fail(cudaStreamSynchronize(s));   // before the vectors are freed
  cudaFree(d_xy);
  return rc;
}

int fz_obs_from_v3_device(int npix, int nw, const float* d_stokes, double* d_obs, void* stream) {
  if (npix <= 0 || nw <= 0 || !d_stokes || !d_obs) return FZ_ERR_ARG;
  k_obs_from_v3<<<grid_for((size_t)npix * nw, 256), 256, 0, (cudaStream_t)stream>>>(npix, nw, d_stokes, d_obs);
  return cuda_fail(cudaGetLastError());
}

int fz_syn_to_v3_device(int npix, int nw, const double* d_syn, float* d_stokes, void* stream) {
  if (npix <= 0 || nw <= 0 || !d_syn || !d_stokes) return FZ_ERR_ARG;
  k_syn_to_v3<<<grid_for((size_t)npix * nw, 256), 256, 0, (cudaStream_t)stream>>>(npix, nw, d_syn, d_stokes);
  return cuda_fail(cudaGetLastError());
}

int fz_rf_to_v3_device(int npix, int nz, int nw, const float* d_rf, float* d_out, void* stream) {
  if (npix <= 0 || nz <= 0 || nw <= 0 || !d_rf || !d_out) return FZ_ERR_ARG;
  if (((uintptr_t)d_out & 7) != 0) return FZ_ERR_ARG;   // float2 stores
  k_rf_to_v3<<<grid_for((size_t)npix * nz * 4 * nw, 256), 256, 0, (cudaStream_t)stream>>>(npix, nz, nw, d_rf, d_out);
  return cuda_fail(cudaGetLastError());
}

int fz_errors_device(fz_ctx* c, int npix, const double* d_obs, const float* d_models, int hydrostatic,
                     const fz_lm_opts* opts, float* d_err, double* d_chi2, int* d_status, void* stream) {
  if (c && c->rf.np > LM_MAXNP) return FZ_ERR_LIMIT;   // errors mode: node layouts of up to 16 nodes
  if (!c || npix <= 0 || !d_obs || !d_models || !d_err || !d_chi2) return FZ_ERR_ARG;
  if (hydrostatic < 0 || hydrostatic > 1) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  LMConf C;
  int rc = lm_conf(c, npix, opts, C);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  static const float kW1[4] = {1.f, 1.f, 1.f, 1.f};
  const std::vector<double> w =
      lm_weights(c->numw, opts ? opts->wstk : kW1, (opts && opts->isigma > 0) ? opts->isigma : 4.0e-3);
  const int nf = C.nfreq, nm = 13 * c->nz;
  // the node Jacobians pass through HBM in chunks of at most 16384 pixels
  // (0.76 GB of REAL*4 EQVDSYN at NP = 13, NFREQ = 896)
  const int chunk = std::min(npix, 16384);
  double *d_w = nullptr, *d_syn = nullptr;
  float *d_jac = nullptr, *d_mout = nullptr;
  int* d_st = nullptr;
  do {
    if ((rc = cuda_fail(cudaMalloc(&d_w, w.size() * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_syn, (size_t)chunk * nf * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_jac, (size_t)chunk * C.np * nf * sizeof(float))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_mout, (size_t)chunk * nm * sizeof(float))))) break;
    if (!d_status && (rc = cuda_fail(cudaMalloc(&d_st, (size_t)chunk * sizeof(int))))) break;
    if ((rc = cuda_fail(cudaMemcpyAsync(d_w, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, s))))
      break;
    const size_t smem = (size_t)c->nz * (sizeof(double) + sizeof(float));
    for (int p0 = 0; p0 < npix && !rc; p0 += chunk) {
      const int n = std::min(chunk, npix - p0);
      int* st = d_status ? d_status + p0 : d_st;
      if ((rc = launch_forward_rf(c, n, d_models + (size_t)p0 * nm, hydrostatic, d_syn, d_jac, d_mout, st, s)))
        break;
      k_lm_errors<<<n, 256, smem, s>>>(C, n, d_obs + (size_t)p0 * nf, d_syn, d_jac, d_mout, d_w, c->d_coef64,
                                       d_err + (size_t)p0 * nm, d_chi2 + p0);
      rc = cuda_fail(cudaGetLastError());
    }
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(s));
  } while (false);
  cudaFree(d_w);
  cudaFree(d_syn);
  cudaFree(d_jac);
  cudaFree(d_mout);
  cudaFree(d_st);
  return rc;
}

int fz_errors(fz_ctx* c, int npix, const double* obs, const float* models, int hydrostatic, const fz_lm_opts* opts,
              float* err, double* chi2, int* status) {
  if (!c || npix <= 0 || !obs || !models || !err || !chi2) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  const size_t nf = 4 * (size_t)c->numw, nm = 13 * (size_t)c->nz;
  cudaStream_t s = c->stream;
  double *d_obs = nullptr, *d_chi = nullptr;
  float *d_m = nullptr, *d_err = nullptr;
  int* d_st = nullptr;
  int rc = 0;
  do {
    if ((rc = cuda_fail(cudaMalloc(&d_obs, npix * nf * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_m, npix * nm * sizeof(float))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_err, npix * nm * sizeof(float))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_chi, npix * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_st, npix * sizeof(int))))) break;
    if ((rc = cuda_fail(cudaMemcpyAsync(d_obs, obs, npix * nf * sizeof(double), cudaMemcpyHostToDevice, s)))) break;
    if ((rc = cuda_fail(cudaMemcpyAsync(d_m, models, npix * nm * sizeof(float), cudaMemcpyHostToDevice, s)))) break;
    if ((rc = fz_errors_device(c, npix, d_obs, d_m, hydrostatic, opts, d_err, d_chi, d_st, s))) break;
    if ((rc = cuda_fail(cudaMemcpyAsync(err, d_err, npix * nm * sizeof(float), cudaMemcpyDeviceToHost, s)))) break;
    if ((rc = cuda_fail(cudaMemcpyAsync(chi2, d_chi, npix * sizeof(double), cudaMemcpyDeviceToHost, s)))) break;
    if (status &&
        (rc = cuda_fail(cudaMemcpyAsync(status, d_st, npix * sizeof(int), cudaMemcpyDeviceToHost, s))))
      break;
    rc = cuda_fail(cudaStreamSynchronize(s));
  } while (false);
  cudaFree(d_obs);
  cudaFree(d_m);
  cudaFree(d_err);
  cudaFree(d_chi);
  cudaFree(d_st);
  return rc;
}

// LSF_INIT's check and upload of one region's kernel (src/pre_post_duties.f90:
// 814-842): valid when |sum(YK) - 1| < 0.01, then YK / sum(YK) once more;
// an invalid region stays unconvolved.  Returns 1 (valid) or 0.
static int lsf_install(fz_ctx* c, int region, std::vector<double>& yk) {
  double sum = 0.0;
  for (double v : yk) sum += v;
  const int valid = std::fabs(sum - 1.0) < 0.01 ? 1 : 0;
  int o = 0;
  for (int r = 0; r < region; ++r) o += c->regs[r].numwave;
  if (c->lsf.yk.size() != (size_t)c->numw) c->lsf.yk.assign(c->numw, 0.0);
  if (valid)
    for (size_t j = 0; j < yk.size(); ++j) c->lsf.yk[o + j] = yk[j] / sum;
  c->lsf.valid[region] = valid;
  FZ_CK(cudaSetDevice(c->device));
  FZ_CK(cudaStreamSynchronize(c->stream));
  if (!c->d_lsf) FZ_CK(cudaMalloc(&c->d_lsf, (size_t)c->numw * sizeof(double)));
  FZ_CK(cudaMemcpy(c->d_lsf, c->lsf.yk.data(), (size_t)c->numw * sizeof(double), cudaMemcpyHostToDevice));
  c->lsf.on = false;
  for (int r = 0; r < c->nreg; ++r) c->lsf.on = c->lsf.on || c->lsf.valid[r];
  return valid;
}

int fz_lsf_gaussian(fz_ctx* c, int region, double sigma, double w0) {
  if (!c || region < 0 || region >= c->nreg || !(sigma > 0.0)) return FZ_ERR_ARG;
  const fz_region& R = c->regs[region];
  const int n = R.numwave;
  if (n < 2) return FZ_ERR_ARG;
  // LSF_INIT's Gaussian (:795-812): pixel positions centred on the region,
  // in mA of WAVE(WI+1) - WAVE(WI), half a step off for even sizes, then
  // normalised and circularly shifted by n/2 (centre to index 0)
  const double dw = (R.wave_ini + R.dlambda * 1.0) - (R.wave_ini + R.dlambda * 0.0);
  std::vector<double> xk(n), yk(n);
  double m = 0.0;
  for (int j = 0; j < n; ++j) {
    xk[j] = (double)(j + 1);
    m += xk[j];
  }
  m /= (double)n;
  for (int j = 0; j < n; ++j) xk[j] = (xk[j] - m) * dw;
  const double woff = (n % 2 == 0) ? (xk[1] - xk[0]) / 2.0 : 0.0;
  double sum = 0.0;
  for (int j = 0; j < n; ++j) {
    const double d = xk[j] - w0 - woff;
    yk[j] = std::exp(-(d * d / (2.0 * sigma * sigma)));
    sum += yk[j];
  }
  std::vector<double> sh(n);
  for (int j = 0; j < n; ++j) sh[j] = yk[(j + n / 2) % n] / sum;
  return lsf_install(c, region, sh);
}

int fz_lsf_kernel(fz_ctx* c, int region, const double* yk, int n) {
  if (!c || region < 0 || region >= c->nreg || !yk) return FZ_ERR_ARG;
  if (n != c->regs[region].numwave) return FZ_ERR_LIMIT;   // READ_LSF_FILE's size check
  std::vector<double> v(yk, yk + n);
  return lsf_install(c, region, v);
}

int fz_lsf_clear(fz_ctx* c) {
  if (!c) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  FZ_CK(cudaStreamSynchronize(c->stream));
  c->lsf.on = false;
  for (int r = 0; r < MAXREG; ++r) c->lsf.valid[r] = 0;
  return 0;
}

int fz_set_tau_device(fz_ctx* c, int nx, int ny, const double* d_obs, float* d_models, int assist, int hydrostatic,
                      void* stream) {
  return fz_set_tau_shard_device(c, nx, ny, d_obs, d_models, assist, hydrostatic, nullptr, nullptr, stream);
}

int fz_set_tau_shard_device(fz_ctx* c, int nx, int ny, const double* d_obs, float* d_models, int assist,
                            int hydrostatic, fz_field_reduce_fn reduce, void* user, void* stream) {
  if (!c || nx <= 0 || ny <= 0 || !d_obs || !d_models || (assist & ~15)) return FZ_ERR_ARG;
  if (assist == 0) return 0;
  const int npix = nx * ny, numw = c->numw, n1 = c->regs[0].numwave, nz = c->nz;
  if (n1 < 3) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  cudaStream_t s = (cudaStream_t)stream;
  double *d_part = nullptr, *d_vec = nullptr, *d_proj = nullptr, *d_syn = nullptr;
  unsigned long long* d_mx = nullptr;
  int rc = 0;
  do {
    if ((rc = cuda_fail(cudaMalloc(&d_part, ((size_t)nx + 1) * n1 * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_vec, (size_t)3 * n1 * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_proj, (size_t)npix * 6 * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_mx, 3 * sizeof(unsigned long long))))) break;
    double* d_tot = d_part + (size_t)nx * n1;
    k_tau_ysum<<<(nx * n1 + 255) / 256, 256, 0, s>>>(nx, ny, numw, n1, d_obs, d_part);
    std::vector<double> v(std::max<size_t>(3 * (size_t)n1, (size_t)nx * n1));
    if (reduce) {
      // a shard of a field split by x: this shard's column sums to the host,
      // the field total (every shard's columns summed in field x order) back
      if ((rc = cuda_fail(cudaMemcpyAsync(v.data(), d_part, (size_t)nx * n1 * sizeof(double), cudaMemcpyDeviceToHost,
                                          s))))
        break;
      if ((rc = cuda_fail(cudaStreamSynchronize(s)))) break;
      if (reduce(user, 0, v.data(), n1, nx) != 0) {
        rc = FZ_ERR_STATE;
        break;
      }
    } else {
      k_tau_xsum<<<(n1 + 127) / 128, 128, 0, s>>>(nx, n1, d_part, d_tot);
      if ((rc = cuda_fail(cudaGetLastError()))) break;
      if ((rc = cuda_fail(cudaMemcpyAsync(v.data(), d_tot, n1 * sizeof(double), cudaMemcpyDeviceToHost, s)))) break;
      if ((rc = cuda_fail(cudaStreamSynchronize(s)))) break;
    }
    std::fill(v.begin() + n1, v.end(), 0.0);
    // VECTORS(:,1..3): the normalised field sum and its two centred
    // derivatives, end points copied, each over SUM(ABS(.)) (:522-534)
    auto norm1 = [&](double* a) {
      double t = 0.0;
      for (int j = 0; j < n1; ++j) t += std::fabs(a[j]);
      for (int j = 0; j < n1; ++j) a[j] = a[j] / t;
    };
    auto deriv = [&](const double* a, double* b) {
      for (int j = 1; j < n1 - 1; ++j) b[j] = (a[j + 1] - a[j - 1]) / 2.0;
      b[0] = b[1];
      b[n1 - 1] = b[n1 - 2];
    };
    double *v1 = v.data(), *v2 = v1 + n1, *v3 = v2 + n1;
    norm1(v1);
    deriv(v1, v2);
    norm1(v2);
    deriv(v2, v3);
    norm1(v3);
    double kol = 0.0;   // KOL = VECTORS(:,2) . VECTORS(:,1) (:613)
    for (int j = 0; j < n1; ++j) kol += v2[j] * v1[j];
    if ((rc = cuda_fail(cudaMemcpyAsync(d_vec, v.data(), 3 * (size_t)n1 * sizeof(double), cudaMemcpyHostToDevice,
                                        s))))
      break;
    const int wblocks = (int)(((size_t)npix * 32 + 255) / 256);
    k_tau_proj<<<wblocks, 256, 0, s>>>(npix, numw, n1, d_obs, d_vec, d_proj);
    if ((rc = cuda_fail(cudaMemsetAsync(d_mx, 0, 3 * sizeof(unsigned long long), s)))) break;
    k_tau_max<<<grid_for(npix, 256), 256, 0, s>>>(npix, kol, d_proj, d_mx);
    if (reduce) {
      // the field maxima over every shard (non-negative doubles)
      unsigned long long hm[3];
      if ((rc = cuda_fail(cudaMemcpyAsync(hm, d_mx, sizeof(hm), cudaMemcpyDeviceToHost, s)))) break;
      if ((rc = cuda_fail(cudaStreamSynchronize(s)))) break;
      double dm[3];
      for (int i = 0; i < 3; ++i) std::memcpy(&dm[i], &hm[i], sizeof(double));
      if (reduce(user, 1, dm, 3, 1) != 0) {
        rc = FZ_ERR_STATE;
        break;
      }
      for (int i = 0; i < 3; ++i) std::memcpy(&hm[i], &dm[i], sizeof(double));
      if ((rc = cuda_fail(cudaMemcpyAsync(d_mx, hm, sizeof(hm), cudaMemcpyHostToDevice, s)))) break;
      if ((rc = cuda_fail(cudaStreamSynchronize(s)))) break;
    }
    TauConf C{};
    C.assist = assist;
    C.nz = nz;
    C.itz = (int)std::ceil((float)nz / 3.0f) - 1;   // CEILING(REAL(NZ)/3.)
    C.kol = kol;
    const double l0 = c->lines[c->regs[0].line[0]].l0;   // LINE_L0(IND_LINE(1)) [A]
    C.lk_hc = (l0 * 1.0e-8 * KBOL) / (HPLA * LIGHT);
    k_tau_apply<<<wblocks, 256, 0, s>>>(C, npix, d_proj, d_mx, d_models);
    if ((rc = cuda_fail(cudaGetLastError()))) break;
    if (assist & 3) {
      // FORWARD3D with HYDRO_TOP off (:675-678): in a hydrostatic run Pg is
      // integrated from the anchor log tau5 = 0 (at ITZ, as just set), then
      // rho, Pe, mu and log tau5 of the new T and Pg
      if ((rc = cuda_fail(cudaMalloc(&d_syn, (size_t)npix * 4 * numw * sizeof(double))))) break;
      if ((rc = launch_forward(c, npix, d_models, hydrostatic ? 2 : 0, d_syn, d_models, nullptr, s))) break;
    }
    rc = cuda_fail(cudaStreamSynchronize(s));
  } while (false);
  cudaFree(d_part);
  cudaFree(d_vec);
  cudaFree(d_proj);
  cudaFree(d_mx);
  cudaFree(d_syn);
  return rc;
}

int fz_set_tau(fz_ctx* c, int nx, int ny, const double* obs, float* models, int assist, int hydrostatic) {
  if (!c || nx <= 0 || ny <= 0 || !obs || !models) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  const size_t npix = (size_t)nx * ny, nf = 4 * (size_t)c->numw, nm = 13 * (size_t)c->nz;
  double* d_obs = nullptr;
  float* d_m = nullptr;
  int rc = 0;
  do {
    if ((rc = cuda_fail(cudaMalloc(&d_obs, npix * nf * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_m, npix * nm * sizeof(float))))) break;
    if ((rc = cuda_fail(cudaMemcpyAsync(d_obs, obs, npix * nf * sizeof(double), cudaMemcpyHostToDevice, c->stream))))
      break;
    if ((rc = cuda_fail(cudaMemcpyAsync(d_m, models, npix * nm * sizeof(float), cudaMemcpyHostToDevice, c->stream))))
      break;
    if ((rc = fz_set_tau_device(c, nx, ny, d_obs, d_m, assist, hydrostatic, c->stream))) break;
    if ((rc = cuda_fail(cudaMemcpyAsync(models, d_m, npix * nm * sizeof(float), cudaMemcpyDeviceToHost, c->stream))))
      break;
    rc = cuda_fail(cudaStreamSynchronize(c->stream));
  } while (false);
  cudaFree(d_obs);
  cudaFree(d_m);
  return rc;
}

int fz_hydrostatic_device(fz_ctx* c, int ncol, const float* d_model, int hydrostatic, float* d_model_out,
                          int* d_status, void* stream) {
  if (!c || ncol <= 0 || !d_model || !d_model_out || hydrostatic < 1 || hydrostatic > 2) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  if (int rc = ensure_scratch(c, ncol)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (d_status) FZ_CK(cudaMemsetAsync(d_status, 0, ncol * sizeof(int), s));
  launch_k_chain(c, ncol, d_model, d_model_out, d_status, hydrostatic, c->tune.chain_warps, c->tune.chain_lanes, s);
  return cuda_fail(cudaGetLastError());
}

int fz_log_tau5_device(fz_ctx* c, int ncol, const float* d_model, int hydrostatic, float* d_model_out, int* d_status,
                       void* stream) {
  if (!c || ncol <= 0 || !d_model || !d_model_out || hydrostatic < 0 || hydrostatic > 2) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  if (int rc = ensure_scratch(c, ncol)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (d_status) FZ_CK(cudaMemsetAsync(d_status, 0, ncol * sizeof(int), s));
  launch_k_chain(c, ncol, d_model, d_model_out, d_status, hydrostatic, c->tune.chain_warps, c->tune.chain_lanes, s);
  FZ_CK(cudaGetLastError());
  const size_t total = (size_t)ncol * c->nz;
  const int blocks = (int)std::min<size_t>((total + 255) / 256, (size_t)c->nsm * 16);
  k_opac<<<blocks, 256, 0, s>>>(c->d_params, c->d_consts, ncol, d_model_out, c->d_chem, c->d_slab);
  k_tau5<<<(ncol + 127) / 128, 128, 0, s>>>(ncol, c->nz, c->sw, c->d_slab, d_model_out);
  return cuda_fail(cudaGetLastError());
}

// the two on host buffers (staging allocated per call)
static int model_only_host(fz_ctx* c, int ncol, const float* model, int hydrostatic, float* model_out, int* status,
                           bool tau) {
  if (!c || ncol <= 0 || !model || !model_out) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  const size_t nm = (size_t)ncol * 13 * c->nz;
  float* d_m = nullptr;
  int* d_st = nullptr;
  int rc = 0;
  do {
    if ((rc = cuda_fail(cudaMalloc(&d_m, nm * sizeof(float))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_st, ncol * sizeof(int))))) break;
    if ((rc = cuda_fail(cudaMemcpyAsync(d_m, model, nm * sizeof(float), cudaMemcpyHostToDevice, c->stream)))) break;
    rc = tau ? fz_log_tau5_device(c, ncol, d_m, hydrostatic, d_m, d_st, c->stream)
             : fz_hydrostatic_device(c, ncol, d_m, hydrostatic, d_m, d_st, c->stream);
    if (rc) break;
    if ((rc = cuda_fail(cudaMemcpyAsync(model_out, d_m, nm * sizeof(float), cudaMemcpyDeviceToHost, c->stream)))) break;
    if (status &&
        (rc = cuda_fail(cudaMemcpyAsync(status, d_st, ncol * sizeof(int), cudaMemcpyDeviceToHost, c->stream))))
      break;
    rc = cuda_fail(cudaStreamSynchronize(c->stream));
  } while (false);
  cudaFree(d_m);
  cudaFree(d_st);
  return rc;
}

int fz_hydrostatic(fz_ctx* c, int ncol, const float* model, int hydrostatic, float* model_out, int* status) {
  return model_only_host(c, ncol, model, hydrostatic, model_out, status, false);
}

int fz_log_tau5(fz_ctx* c, int ncol, const float* model, int hydrostatic, float* model_out, int* status) {
  return model_only_host(c, ncol, model, hydrostatic, model_out, status, true);
}

int fz_smooth(fz_ctx* c, int nx, int ny, float* models, const int* params) {
  if (!c || nx <= 0 || ny <= 0 || !models) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  const size_t bytes = (size_t)nx * ny * 13 * c->nz * sizeof(float);
  float* d = nullptr;
  FZ_CK(cudaMalloc(&d, bytes));
  int rc = cuda_fail(cudaMemcpyAsync(d, models, bytes, cudaMemcpyHostToDevice, c->stream));
  if (!rc) rc = fz_smooth_device(c, nx, ny, d, params, c->stream);
  if (!rc) rc = cuda_fail(cudaMemcpyAsync(models, d, bytes, cudaMemcpyDeviceToHost, c->stream));
  if (!rc) rc = cuda_fail(cudaStreamSynchronize(c->stream));
  cudaFree(d);
  return rc;
}

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
  Consts K;
  host_consts(K);
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
    P.cont[r] = host_cont(main.l0);
    for (int b = 0; b < R.nblend; ++b) {
      if (R.line[b] < 0 || R.line[b] >= nlines || nlu >= MAXLU) {
        delete c;
        return nlu >= MAXLU ? FZ_ERR_LIMIT : FZ_ERR_ARG;
      }
      const fz_line& L = lines[R.line[b]];
      P.lu[nlu] = host_line(L, b == 0 ? 0.0 : R.wdif[b], K);
      P.lu_duv[nlu] = (float)(-1e3 * L.l0 / LIGHT);
      std::vector<double> sh, stg;
      std::vector<int> ty;
      const int n = fzh_zeeman(L, sh, stg, ty);
      if (n < 0 || ncomp + n > MAXCOMP) {
        delete c;
        return n < 0 ? FZ_ERR_ARG : FZ_ERR_LIMIT;
      }
      P.lu_c0[nlu] = ncomp;
      int at = ncomp;
      // group by type (ZEEMAN_COMP order kept within a type); components of
      // zero strength (the M = 0 -> 0 pi component of a Delta J = 0 line) add
      // exactly nothing to any sum and are left out
      for (int t = -1; t <= 1; ++t) {
        P.lu_nt[nlu][t + 1] = 0;
        for (int i = 0; i < n; ++i)
          if (ty[i] == t && stg[i] != 0.0) {
            P.comp_shift[at] = (float)sh[i];
            P.comp_str[at] = (float)stg[i];
            P.comp_type[at] = t;
            ++at;
            ++P.lu_nt[nlu][t + 1];
          }
      }
      P.lu_nc[nlu] = at - ncomp;
      ncomp = at;
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
  P.cont[nreg] = host_cont(5000.0);   // KC5 (src/forward.f90:926)
  c->numw = numw;
  c->nlu = nlu;
  c->sw = slab_w(nreg, nlu);
  P.nz = nz;
  P.numw = numw;
  P.nreg = nreg;
  P.nlu = nlu;
  P.sw = c->sw;
  int rc = 0;
  auto fail = [&](int code) {
    fz_destroy(c);
    return code;
  };
  if ((rc = cuda_fail(cudaSetDevice(device)))) return fail(rc);
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
  if ((rc = cuda_fail(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)))) return fail(rc);
  if ((rc = cuda_fail(cudaMalloc(&c->d_params, sizeof(DevParams))))) return fail(rc);
  if ((rc = cuda_fail(cudaMalloc(&c->d_consts, sizeof(Consts))))) return fail(rc);
  if ((rc = cuda_fail(cudaMalloc(&c->d_pf, sizeof(PFTable))))) return fail(rc);
  {
    std::vector<char> buf(sizeof(PFTable));
    fzh_pf_table(reinterpret_cast<PFTable*>(buf.data()));
    if ((rc = cuda_fail(cudaMemcpy(c->d_pf, buf.data(), sizeof(PFTable), cudaMemcpyHostToDevice)))) return fail(rc);
  }
  if ((rc = cuda_fail(cudaMalloc(&c->d_pfd, sizeof(PFDTable))))) return fail(rc);
  {
    std::vector<char> buf(sizeof(PFDTable));
    if (fzh_pfd_table(reinterpret_cast<PFDTable*>(buf.data())) != 0) return fail(FZ_ERR_STATE);
    if ((rc = cuda_fail(cudaMemcpy(c->d_pfd, buf.data(), sizeof(PFDTable), cudaMemcpyHostToDevice)))) return fail(rc);
  }
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
    k_gain<<<1, 256, FZ_HSRA_LEN * nreg * sizeof(double), c->stream>>>(c->d_params, c->d_consts, c->d_pf, d_l,
                                                                        c->d_gain, d_st);
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

int fz_measure_fp64_peak(int device, double* tflops) {
  if (!tflops) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(device));
  int sms = 0;
  FZ_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  double* d = nullptr;
  FZ_CK(cudaMalloc(&d, sizeof(double)));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int threads = 512, blocks = sms * 4, iters = 16;
  k_fp64_peak<<<blocks, threads>>>(d, iters, 1e-9);   // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(a);
    k_fp64_peak<<<blocks, threads>>>(d, iters, 1e-9);
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
  const double fma = (double)blocks * threads * iters * 32 * 8;
  *tflops = 2.0 * fma / (best * 1e-3) / 1e12;
  return 0;
}

int fz_destroy(fz_ctx* c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->d_params);
  cudaFree(c->d_consts);
  cudaFree(c->d_pf);
  cudaFree(c->d_pfd);
  cudaFree(c->d_oscr);
  cudaFree(c->d_smooth);
  cudaFree(c->d_lsf);
  for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
  for (auto& p : c->pending) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (void* p : {(void*)c->inv.obs, (void*)c->inv.chi, (void*)c->inv.syn, (void*)c->inv.tgt, (void*)c->inv.init,
                  (void*)c->inv.out, (void*)c->inv.it, (void*)c->inv.st, (void*)c->inv.fb})
    cudaFree(p);
  cudaFree(c->d_lam);
  cudaFree(c->d_gain);
  cudaFree(c->d_slab);
  cudaFree(c->d_chem);
  cudaFree(c->d_saha);
  cudaFree(c->d_model);
  cudaFree(c->d_syn);
  cudaFree(c->d_status);
  cudaFree(c->d_rf);
  cudaFree(c->d_coef);
  cudaFree(c->d_rfslab);
  cudaFree(c->d_chemd);
  cudaFree(c->d_jac);
  cudaFree(c->d_coef64);
  cudaFree(c->inv.state);
  cudaFree(c->d_rfbig);
  cudaFree(c->d_nrow);
  cudaFree(c->d_nnorm);
  cudaFree(c->d_nhss);
  cudaFree(c->d_svd);
  cudaFree(c->d_wsy);
  cudaFree(c->d_wsnorm);
  lm_free(c);
  cudaFree(c->d_q);
  if (c->h_done) cudaFreeHost(c->h_done);
  if (c->h_q) cudaFreeHost(c->h_q);
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

int fz_profile_read(fz_ctx* c, double* ms, int* launches, long long* items, int n) {
  if (!c) return FZ_ERR_ARG;
  for (auto& p : c->pending) {
    float t = 0.f;
    if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) {
      c->prof_ms[p.kernel] += t;
      c->prof_n[p.kernel] += 1;
    }
    c->ev_pool.push_back(p.a);
    c->ev_pool.push_back(p.b);
  }
  c->pending.clear();
  for (int i = 0; i < n && i < NKERN; ++i) {
    if (ms) ms[i] = c->prof_ms[i];
    if (launches) launches[i] = c->prof_n[i];
    if (items) items[i] = c->prof_items[i];
    c->prof_ms[i] = 0;
    c->prof_n[i] = 0;
    c->prof_items[i] = 0;
  }
  return NKERN;
}

int fz_get_gain(fz_ctx* c, float* gain) {
  if (!c || !gain) return FZ_ERR_ARG;
  std::memcpy(gain, c->gain.data(), c->gain.size() * sizeof(float));
  return 0;
}

int fz_forward_device(fz_ctx* c, int ncol, const float* d_model, int hydrostatic, double* d_syn,
                      float* d_model_out, int* d_status, void* stream) {
  if (!c || ncol <= 0 || !d_model || !d_syn || !d_model_out) return FZ_ERR_ARG;
  if (hydrostatic < 0 || hydrostatic > 2) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  return launch_forward(c, ncol, d_model, hydrostatic, d_syn, d_model_out, d_status, (cudaStream_t)stream);
}

int fz_rf_nodes(fz_ctx* c, const int* nodes) {
  if (!c || !nodes) return FZ_ERR_ARG;
  // reference parameter (1-based) of each slot; rho (3) and P0 (8) are not supported
  static const int kRef[NSLOT] = {1, 2, 4, 5, 6, 7};
  if (nodes[2] != 0 || nodes[7] != 0) return FZ_ERR_ARG;
  RFConf rf{};
  int np = 0;
  for (int p = 0; p < NSLOT; ++p) {
    const int nj = nodes[kRef[p] - 1];
    if (nj < 0 || nj > c->nz) return FZ_ERR_ARG;
    rf.n0[p] = np;
    rf.nj[p] = nj;
    np += nj;
  }
  if (np <= 0) return FZ_ERR_ARG;
  if (np > LM_MAXNP_BIG) return FZ_ERR_LIMIT;
  rf.np = np;
  std::vector<float> tab((size_t)c->nz * np, 0.0f);
  std::vector<double> cf;
  for (int p = 0; p < NSLOT; ++p) {
    if (rf.nj[p] == 0) continue;
    int_coefs(c->nz, rf.nj[p], cf);
    for (int j = 0; j < rf.nj[p]; ++j)
      for (int k = 0; k < c->nz; ++k) tab[(size_t)k * np + rf.n0[p] + j] = (float)cf[(size_t)j * c->nz + k];
  }
  c->rf.np = 0;
  FZ_CK(cudaSetDevice(c->device));
  FZ_CK(cudaStreamSynchronize(c->stream));
  cudaFree(c->d_coef);
  c->d_coef = nullptr;
  if (!c->d_rf) FZ_CK(cudaMalloc(&c->d_rf, sizeof(RFConf)));
  FZ_CK(cudaMalloc(&c->d_coef, tab.size() * sizeof(float)));
  FZ_CK(cudaMemcpy(c->d_coef, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice));
  {
    std::vector<double> t64((size_t)c->nz * np, 0.0);
    for (int p = 0; p < NSLOT; ++p) {
      if (rf.nj[p] == 0) continue;
      int_coefs(c->nz, rf.nj[p], cf);
      for (int j = 0; j < rf.nj[p]; ++j)
        for (int k = 0; k < c->nz; ++k) t64[(size_t)k * np + rf.n0[p] + j] = cf[(size_t)j * c->nz + k];
    }
    cudaFree(c->d_coef64);
    c->d_coef64 = nullptr;
    FZ_CK(cudaMalloc(&c->d_coef64, t64.size() * sizeof(double)));
    FZ_CK(cudaMemcpy(c->d_coef64, t64.data(), t64.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  FZ_CK(cudaMemcpy(c->d_rf, &rf, sizeof(RFConf), cudaMemcpyHostToDevice));
  {
    // per-node model rows and PARAM_NORMS for the large-layout LM kernels
    static const int kRow[9] = {0, 0, 1, 2, 5, 6, 7, 10, 1};
    const double norms[8] = {6000.0, 1.0e5, 1.0e-5, 1.0e3, 1.0e3, 1.0e3, 1.0e6, 6.0e2};
    std::vector<int> row(np);
    std::vector<double> nrm(np);
    for (int p = 0; p < NSLOT; ++p)
      for (int j = 0; j < rf.nj[p]; ++j) {
        row[rf.n0[p] + j] = kRow[kRef[p]];
        nrm[rf.n0[p] + j] = norms[kRef[p] - 1];
      }
    cudaFree(c->d_nrow);
    cudaFree(c->d_nnorm);
    c->d_nrow = nullptr;
    c->d_nnorm = nullptr;
    FZ_CK(cudaMalloc(&c->d_nrow, np * sizeof(int)));
    FZ_CK(cudaMalloc(&c->d_nnorm, np * sizeof(double)));
    FZ_CK(cudaMemcpy(c->d_nrow, row.data(), np * sizeof(int), cudaMemcpyHostToDevice));
    FZ_CK(cudaMemcpy(c->d_nnorm, nrm.data(), np * sizeof(double), cudaMemcpyHostToDevice));
    c->nhss_host.clear();
  }
  c->rf = rf;
  const size_t sms = rf_smem(c);
  int maxsm = 0;
  FZ_CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
  // the forward accumulation keeps 4 x NP accumulators per wavelength in
  // shared memory; larger layouts contract the full response functions
  c->rf_full = sms > (size_t)maxsm || np > MAXNP;
  if (c->rf_full) return np;
  FZ_CK((set_synth_rf_attr<true, false>(cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sms)));
  FZ_CK((set_synth_rf_attr<false, false>(cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sms)));
  // all of the SM's unified L1/shared storage as shared memory: two CTAs of
  // ~90 KB each can then be resident
  FZ_CK((set_synth_rf_attr<true, false>(cudaFuncAttributePreferredSharedMemoryCarveout, 100)));
  FZ_CK((set_synth_rf_attr<false, false>(cudaFuncAttributePreferredSharedMemoryCarveout, 100)));
  return np;
}

int fz_forward_rf_device(fz_ctx* c, int ncol, const float* d_model, int hydrostatic, double* d_syn, float* d_jac,
                         float* d_model_out, int* d_status, void* stream) {
  if (!c || ncol <= 0 || !d_model || !d_syn || !d_jac || !d_model_out) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  return launch_forward_rf(c, ncol, d_model, hydrostatic, d_syn, d_jac, d_model_out, d_status, (cudaStream_t)stream);
}

int fz_invert_device(fz_ctx* c, int npix, const double* d_obs, const float* d_init, const double* d_target_chi2,
                     int hydrostatic, const fz_lm_opts* opts, float* d_model_out, double* d_chi2, int* d_iters,
                     double* d_syn_out, int* d_status, void* stream) {
  if (!c || npix <= 0 || !d_obs || !d_init || !d_model_out || !d_chi2 || !d_iters) return FZ_ERR_ARG;
  if (hydrostatic < 0 || hydrostatic > 1) return FZ_ERR_ARG;
  if (int rc = rf_check(c)) return rc;
  FZ_CK(cudaSetDevice(c->device));
  LMConf C;
  int rc = lm_conf(c, npix, opts, C);
  if (rc) return rc;
  int S = (opts && opts->slots > 0) ? opts->slots : c->tune.lm_slots;
  if (C.global_stop) S = npix;   // the field rule needs every pixel in flight
  if (S > npix) S = npix;
  const bool big = C.np > LM_MAXNP;
  if (big) {
    // large layouts: the slot count within a memory budget (Jacobian, H and
    // SVD scratch per slot and pool, full response functions and operators)
    const size_t nf = 4 * (size_t)c->numw, np = C.np;
    const size_t per = 2 * (np * nf * 4 + np * np * 8) + 2 * np * np * 8 + (size_t)NSLOT * c->nz * nf * 4 +
                       (size_t)c->nz * 16 * c->numw * 4;
    const size_t cap = std::max<size_t>(1, ((size_t)24 << 30) / per);
    if ((size_t)S > cap) {
      if (C.global_stop) return FZ_ERR_LIMIT;
      S = (int)cap;
    }
  }
  if ((rc = lm_alloc(c, S))) return rc;
  if (big) {
    if (C.solver != 2) {
      const size_t need = (size_t)S * 2 * C.np * C.np;
      if (need > c->svd_len) {
        cudaFree(c->d_svd);
        c->d_svd = nullptr;
        c->svd_len = 0;
        FZ_CK(cudaMalloc(&c->d_svd, need * sizeof(double)));
        c->svd_len = need;
      }
    }
    FZ_CK(cudaFuncSetAttribute(k_lm_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GT_SMEM));
  }
  // The iterations run on the context's own stream (capturable, unlike a
  // caller's legacy default stream), after the work already enqueued on the
  // caller's stream; the call returns with everything complete.
  cudaStream_t s = c->stream;
  {
    cudaEvent_t ev = nullptr;
    FZ_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    const cudaError_t e1 = cudaEventRecord(ev, (cudaStream_t)stream);
    const cudaError_t e2 = e1 == cudaSuccess ? cudaStreamWaitEvent(s, ev, 0) : e1;
    cudaEventDestroy(ev);
    FZ_CK(e2);
  }
  if (!c->d_q) FZ_CK(cudaMalloc(&c->d_q, sizeof(LMQueue)));
  if (!c->h_done) FZ_CK(cudaMallocHost(&c->h_done, sizeof(int)));
  static const float kW1[4] = {1.f, 1.f, 1.f, 1.f};
  const std::vector<double> w =
      lm_weights(c->numw, opts ? opts->wstk : kW1, (opts && opts->isigma > 0) ? opts->isigma : 4.0e-3);
  double* d_w = nullptr;
  FZ_CK(cudaMalloc(&d_w, w.size() * sizeof(double)));
  struct Free {
    double* p;
    ~Free() { cudaFree(p); }
  } fw{d_w};
  FZ_CK(cudaMemcpyAsync(d_w, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  FZ_CK(cudaMemsetAsync(c->d_q, 0, sizeof(LMQueue), s));
  if (d_status) FZ_CK(cudaMemsetAsync(d_status, 0, npix * sizeof(int), s));
  LMSlots L = c->lm, L2 = c->lm2;   // L is the pool in use; it shrinks to the occupied slots in the tail
  if (!C.reg) L.pen = L2.pen = nullptr;
  {
    ProfScope ps(c, 5, s, S);
    k_lm_fill<<<S, 128, 0, s>>>(C, L, c->d_q, d_obs, d_init);
  }
  FZ_CK(cudaGetLastError());
  const size_t usm = (size_t)(C.nz + 3 * C.np) * sizeof(double) + (size_t)C.nz * sizeof(float);
  LMQueue hq{};
  // every pixel needs at most maxit iterations; slots are refilled at once
  const long long cap = (long long)C.maxit * ((npix + S - 1) / S + 1) + 8;
  if (!c->h_q) FZ_CK(cudaMallocHost(&c->h_q, sizeof(LMQueue)));
  if ((rc = ensure_rf_scratch(c, S))) return rc;
  // one LM iteration over the n slots of pool L: synthesis of the current
  // models, accept/refill, the response functions of the accepted models of
  // pixels that go on (into the best Jacobian), normal equations, solve,
  // update, and the queue state to the host
  auto iteration = [&](int n) -> int {
    int r = launch_forward(c, n, L.mcur, hydrostatic, L.syn, L.mcur, L.status, s);
    if (r) return r;
    {
      ProfScope ps(c, 6, s, n);
      k_lm_accept<<<n, 256, C.reg ? 2 * C.np * sizeof(double) : 0, s>>>(C, L, c->d_q, d_w, d_obs, d_init,
                                                                        d_target_chi2, d_model_out, d_chi2, d_iters,
                                    d_syn_out, d_status, c->d_coef64);
    }
    k_lm_rflist<<<1, 1024, 0, s>>>(n, L.need_rf, L.rf_list, c->d_q);
    FZ_CK(cudaGetLastError());
    r = launch_rf_stage(c, n, hydrostatic, L.syn, L.jacb, L.mcur, L.status, s, L.rf_list, &c->d_q->rf_count);
    if (r) return r;
    if (big) {
      // tcgen05 normal equations over tile pairs, FP64 gradient, CTA solver
      const int nb = (C.np + GT_M - 1) / GT_M;
      {
        ProfScope ps(c, 7, s, n);
        k_lm_gram_tc<<<dim3(nb * (nb + 1) / 2, n), 128, GT_SMEM, s>>>(C, L, d_w, &c->d_q->tc_err);
        k_lm_grad<<<dim3((C.np + 7) / 8, n), 256, 0, s>>>(C, L, d_w);
      }
      {
        ProfScope ps(c, 8, s, n);
        if (C.solver == 2)
          k_lm_cg_big<<<n, 256, 6 * C.np * sizeof(double), s>>>(C, L);
        else
          k_lm_svd_big<<<n, 256, 2 * C.np * sizeof(double), s>>>(C, L, c->d_svd);
      }
    } else {
      {
        ProfScope ps(c, 7, s, n);
        k_lm_normal<<<(n + 3) / 4, 128, 0, s>>>(C, L, d_w, L.rf_list, &c->d_q->rf_count);
      }
      {
        ProfScope ps(c, 8, s, n);
        k_lm_solve<<<(n + 3) / 4, 128, 0, s>>>(C, L);
      }
    }
    {
      ProfScope ps(c, 9, s, n);
      k_lm_update<<<n, 128, usm, s>>>(C, L, c->d_coef64);
    }
    k_lm_scan<<<1, 1024, 0, s>>>(n, L.pix, c->d_dest, c->d_q);
    FZ_CK(cudaGetLastError());
    FZ_CK(cudaMemcpyAsync(c->h_q, c->d_q, sizeof(LMQueue), cudaMemcpyDeviceToHost, s));
    return 0;
  };
  // Without profiling, the iteration is captured once per pool state (slot
  // count and pool) as a CUDA graph and replayed until a compaction changes
  // it; with profiling, its kernels are launched one by one between events.
  struct Graph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    void reset() {
      if (e) cudaGraphExecDestroy(e);
      if (g) cudaGraphDestroy(g);
      e = nullptr;
      g = nullptr;
    }
    ~Graph() { reset(); }
  } graph;
  // The device-driven loop (no per-kernel profiling, node layouts of the
  // warp kernels, no LSF): one CUDA graph whose WHILE node repeats an
  // iteration over the occupied slots of the whole pool until k_lm_ctl --
  // the last node of the body -- finds the queue done, the iteration cap
  // reached or the field-wide stop met.  The synthesis kernels walk the list
  // of occupied slots the previous iteration's scan wrote (a finished pixel's
  // slot takes the next pixel at once; once the queue is drained the list
  // shrinks instead of the pool being compacted), the response functions
  // the list of accepted slots; the host launches the graph once and reads
  // the queue state once.
  if (!c->prof && !big && !c->lsf.on) {
    if ((rc = ensure_scratch(c, S))) return rc;
    const int gthr = C.global_stop ? std::max(1, C.maxsteps - opts->cycles_left) : 0;
    k_lm_scan<<<1, 1024, 0, s>>>(S, L.pix, c->d_dest, c->d_q, c->d_act);   // the filled slots
    FZ_CK(cudaGetLastError());
    struct Loop {
      cudaGraph_t g = nullptr;
      cudaGraphExec_t e = nullptr;
      ~Loop() {
        if (e) cudaGraphExecDestroy(e);
        if (g) cudaGraphDestroy(g);
      }
    } loop;
    FZ_CK(cudaGraphCreate(&loop.g, 0));
    cudaGraphConditionalHandle h = 0;
    FZ_CK(cudaGraphConditionalHandleCreate(&h, loop.g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    FZ_CK(cudaGraphAddNode(&node, loop.g, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    FZ_CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int r = launch_forward(c, S, L.mcur, hydrostatic, L.syn, L.mcur, L.status, s, c->d_act, &c->d_q->active);
    if (!r) {
      k_lm_accept<<<S, 256, C.reg ? 2 * C.np * sizeof(double) : 0, s>>>(C, L, c->d_q, d_w, d_obs, d_init,
                                                                       d_target_chi2, d_model_out, d_chi2, d_iters,
                                                                       d_syn_out, d_status, c->d_coef64);
      k_lm_rflist<<<1, 1024, 0, s>>>(S, L.need_rf, L.rf_list, c->d_q);
      r = launch_rf_stage(c, S, hydrostatic, L.syn, L.jacb, L.mcur, L.status, s, L.rf_list, &c->d_q->rf_count);
    }
    if (!r) {
      k_lm_normal<<<(S + 3) / 4, 128, 0, s>>>(C, L, d_w, L.rf_list, &c->d_q->rf_count);
      k_lm_solve<<<(S + 3) / 4, 128, 0, s>>>(C, L);
      k_lm_update<<<S, 128, usm, s>>>(C, L, c->d_coef64);
      k_lm_scan<<<1, 1024, 0, s>>>(S, L.pix, c->d_dest, c->d_q, c->d_act);
      k_lm_ctl<<<1, 1, 0, s>>>(c->d_q, h, npix, cap, gthr);
    }
    cudaGraph_t captured = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &captured);
    if (r) return r;
    FZ_CK(ce);
    FZ_CK(cudaGraphInstantiate(&loop.e, loop.g, 0));
    FZ_CK(cudaGraphLaunch(loop.e, s));
    FZ_CK(cudaMemcpyAsync(c->h_q, c->d_q, sizeof(LMQueue), cudaMemcpyDeviceToHost, s));
    FZ_CK(cudaStreamSynchronize(s));
    hq = *c->h_q;
    if (hq.tc_err) {
      std::fprintf(stderr, "fz_b200: the tensor-core normal equations gave up waiting for their MMAs\n");
      return FZ_ERR_CUDA;
    }
    if (hq.gstop) {
      k_lm_finish_all<<<S, 256, 0, s>>>(C, L, c->d_q, d_model_out, d_chi2, d_iters, d_syn_out, d_status);
      FZ_CK(cudaGetLastError());
      FZ_CK(cudaStreamSynchronize(s));
      return 0;
    }
    return hq.done >= npix ? 0 : FZ_ERR_STATE;
  }
  int graph_n = -1;
  const float* graph_pool = nullptr;
  for (long long it = 0; it < cap; ++it) {
    const int n = L.S;
    if (c->prof) {
      if ((rc = iteration(n))) return rc;
    } else {
      if (!graph.e || graph_n != n || graph_pool != L.mcur) {
        graph.reset();
        FZ_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        rc = iteration(n);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(s, &g);
        graph.g = g;
        if (rc) return rc;
        FZ_CK(ce);
        FZ_CK(cudaGraphInstantiate(&graph.e, graph.g, 0));
        graph_n = n;
        graph_pool = L.mcur;
      }
      FZ_CK(cudaGraphLaunch(graph.e, s));
    }
    FZ_CK(cudaStreamSynchronize(s));
    hq = *c->h_q;
    if (hq.tc_err) {
      std::fprintf(stderr, "fz_b200: the tensor-core normal equations gave up waiting for their MMAs\n");
      return FZ_ERR_CUDA;
    }
    if (c->prof) {   // columns of the RF pass: known once the iteration ran
      c->prof_items[10] += hq.rf_count;
      c->prof_items[3] += hq.rf_count;
      c->prof_items[4] += hq.rf_count;
    }
    if (hq.done >= npix) return 0;
    if (C.global_stop) {
      // MAKE_DECISION: the field stops once the mean STEPS over its pixels
      // reaches max(1, MAXSTEPS - (MAXITER - CURIC))
      const int thr = std::max(1, C.maxsteps - opts->cycles_left);
      if ((double)(long long)hq.steps_sum >= (double)thr * (double)npix) {
        k_lm_finish_all<<<n, 256, 0, s>>>(C, L, c->d_q, d_model_out, d_chi2, d_iters, d_syn_out, d_status);
        FZ_CK(cudaGetLastError());
        FZ_CK(cudaStreamSynchronize(s));
        return 0;
      }
    }
    // the queue is drained: move the occupied slots to the front of the
    // other pool once a quarter of the pool has emptied, and iterate on them only
    if (hq.next >= npix && hq.active > 0 && hq.active <= (3 * n) / 4) {
      k_lm_compact<<<n, 256, 0, s>>>(C, L, L2, c->d_dest);
      FZ_CK(cudaGetLastError());
      std::swap(L, L2);
      L.S = hq.active;
      L2.S = S;
    }
  }
  return FZ_ERR_STATE;
}

static void inv_free(fz_ctx* c) {
  cudaFree(c->inv.obs);
  cudaFree(c->inv.chi);
  cudaFree(c->inv.syn);
  cudaFree(c->inv.tgt);
  cudaFree(c->inv.init);
  cudaFree(c->inv.out);
  cudaFree(c->inv.it);
  cudaFree(c->inv.st);
  cudaFree(c->inv.fb);
  cudaFree(c->inv.state);
  c->inv = {};
}

int fz_invert(fz_ctx* c, int npix, const double* obs, const float* init, const double* target_chi2, int hydrostatic,
              const fz_lm_opts* opts, float* model_out, double* chi2, int* iters, double* syn_out, int* status) {
  if (!c || npix <= 0 || !obs || !init || !model_out || !chi2 || !iters) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  const size_t nf = 4 * (size_t)c->numw, nm = 13 * (size_t)c->nz;
  cudaStream_t s = c->stream;
  // device staging kept in the context between calls; it grows when a call
  // brings more pixels (or asks for the synthesis for the first time)
  if ((size_t)npix > c->inv.cap || (syn_out && !c->inv.has_syn)) {
    FZ_CK(cudaStreamSynchronize(s));
    const size_t n = std::max((size_t)npix, c->inv.cap);
    const bool ws = syn_out || c->inv.has_syn;
    inv_free(c);
    int rc = 0;
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.obs, n * nf * sizeof(double)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.init, n * nm * sizeof(float)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.out, n * nm * sizeof(float)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.chi, n * sizeof(double)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.tgt, n * sizeof(double)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.it, n * sizeof(int)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.st, n * sizeof(int)));
    if (!rc && ws) rc = cuda_fail(cudaMalloc(&c->inv.syn, n * nf * sizeof(double)));
    if (rc) {
      inv_free(c);
      return rc;
    }
    c->inv.cap = n;
    c->inv.has_syn = ws;
  }
  FZ_CK(cudaMemcpyAsync(c->inv.obs, obs, npix * nf * sizeof(double), cudaMemcpyHostToDevice, s));
  FZ_CK(cudaMemcpyAsync(c->inv.init, init, npix * nm * sizeof(float), cudaMemcpyHostToDevice, s));
  if (target_chi2)
    FZ_CK(cudaMemcpyAsync(c->inv.tgt, target_chi2, npix * sizeof(double), cudaMemcpyHostToDevice, s));
  // the fallback model comes from host memory here
  fz_lm_opts o{};
  if (opts) o = *opts;
  if (opts && opts->fallback_model) {
    if (!c->inv.fb) FZ_CK(cudaMalloc(&c->inv.fb, nm * sizeof(float)));
    FZ_CK(cudaMemcpyAsync(c->inv.fb, opts->fallback_model, nm * sizeof(float), cudaMemcpyHostToDevice, s));
    o.fallback_model = c->inv.fb;
  }
  if (opts && opts->state_out) {
    if ((size_t)npix > c->inv.state_cap) {
      cudaFree(c->inv.state);
      c->inv.state = nullptr;
      c->inv.state_cap = 0;
      FZ_CK(cudaMalloc(&c->inv.state, (size_t)npix * 5 * sizeof(double)));
      c->inv.state_cap = npix;
    }
    o.state_out = c->inv.state;
  }
  int rc = fz_invert_device(c, npix, c->inv.obs, c->inv.init, target_chi2 ? c->inv.tgt : nullptr, hydrostatic,
                            opts ? &o : nullptr,
                            c->inv.out, c->inv.chi, c->inv.it, syn_out ? c->inv.syn : nullptr, c->inv.st, s);
  if (rc) return rc;
  FZ_CK(cudaMemcpyAsync(model_out, c->inv.out, npix * nm * sizeof(float), cudaMemcpyDeviceToHost, s));
  FZ_CK(cudaMemcpyAsync(chi2, c->inv.chi, npix * sizeof(double), cudaMemcpyDeviceToHost, s));
  FZ_CK(cudaMemcpyAsync(iters, c->inv.it, npix * sizeof(int), cudaMemcpyDeviceToHost, s));
  if (status) FZ_CK(cudaMemcpyAsync(status, c->inv.st, npix * sizeof(int), cudaMemcpyDeviceToHost, s));
  if (syn_out) FZ_CK(cudaMemcpyAsync(syn_out, c->inv.syn, npix * nf * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (opts && opts->state_out)
    FZ_CK(cudaMemcpyAsync(opts->state_out, c->inv.state, (size_t)npix * 5 * sizeof(double), cudaMemcpyDeviceToHost,
                          s));
  FZ_CK(cudaStreamSynchronize(s));
  return 0;
}

// Batched GET_PERTURBATION on host buffers; the Jacobian comes as REAL*8
// (jac64) or REAL*4 (jac32), exactly one of them given.  A REAL*8 Jacobian is
// rounded to FP32 on the device before the split-bf16 normal equations.
static int lm_perturbation_host(fz_ctx* c, int npix, int np, int nfreq, const double* jac64, const float* jac32,
                                const double* diff, const double* lambda, const double* reg_pen,
                                const double* reg_hss, int dtype, double svdtol, double* delta) {
  if (!c || npix <= 0 || np <= 0 || np > LM_MAXNP_BIG || nfreq <= 0 || (nfreq & 3) || (!jac64 == !jac32) || !diff || !lambda || !delta)
    return FZ_ERR_ARG;
  if (dtype < 0 || dtype > 2) return FZ_ERR_ARG;   // GET_PERTURBATION's DTYPE (0 taken as 1)
  FZ_CK(cudaSetDevice(c->device));
  LMConf C;
  std::memset(&C, 0, sizeof(C));
  C.np = np;
  C.nfreq = nfreq;
  C.inu = 1.0;
  C.svdtol = svdtol > 0 ? svdtol : 1.0e-4;
  C.solver = dtype == 2 ? 2 : 1;
  const bool big = np > LM_MAXNP;
  for (int j = 0; j < np && !big; ++j) C.norm[j] = 1.0;
  double* d_ones = nullptr;   // PARAM_NORMS of a large layout: the Jacobian comes normalised
  int* d_err = nullptr;
  double* d_svd = nullptr;
  LMSlots L{};
  L.S = npix;
  std::vector<int> zeros(npix, 0);
  std::vector<double> st(5 * (size_t)npix, 0.0);
  for (int i = 0; i < npix; ++i) st[5 * (size_t)i + 2] = lambda[i];
  std::vector<double> ones(nfreq, 1.0);
  double* d_w = nullptr;
  int rc = 0;
  do {
    if ((rc = cuda_fail(cudaMalloc(&L.pix, npix * sizeof(int))))) break;
    if ((rc = cuda_fail(cudaMalloc(&L.skip, npix * sizeof(int))))) break;
    if ((rc = cuda_fail(cudaMalloc(&L.st, st.size() * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&L.jacb, (size_t)npix * np * nfreq * sizeof(float))))) break;
    if ((rc = cuda_fail(cudaMalloc(&L.diff, (size_t)npix * nfreq * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&L.H, (size_t)npix * np * np * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&L.g, (size_t)npix * np * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&L.delta, (size_t)npix * np * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_w, nfreq * sizeof(double))))) break;
    if (big) {
      std::vector<double> ones(np, 1.0);
      if ((rc = cuda_fail(cudaMalloc(&d_ones, np * sizeof(double))))) break;
      if ((rc = cuda_fail(cudaMalloc(&d_err, sizeof(int))))) break;
      if (C.solver != 2 && (rc = cuda_fail(cudaMalloc(&d_svd, (size_t)npix * 2 * np * np * sizeof(double))))) break;
      cudaMemcpy(d_ones, ones.data(), np * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemset(d_err, 0, sizeof(int));
      C.d_norm = d_ones;
    }
    if (reg_pen) {
      if ((rc = cuda_fail(cudaMalloc(&L.pen, (size_t)npix * np * sizeof(double))))) break;
      cudaMemcpy(L.pen, reg_pen, (size_t)npix * np * sizeof(double), cudaMemcpyHostToDevice);
    }
    if (reg_hss) {
      if ((rc = cuda_fail(cudaMalloc(&L.hss, (size_t)npix * np * np * sizeof(double))))) break;
      cudaMemcpy(L.hss, reg_hss, (size_t)npix * np * np * sizeof(double), cudaMemcpyHostToDevice);
    }
    cudaMemcpy(L.pix, zeros.data(), npix * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(L.skip, zeros.data(), npix * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(L.st, st.data(), st.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (jac32) {
      cudaMemcpy(L.jacb, jac32, (size_t)npix * np * nfreq * sizeof(float), cudaMemcpyHostToDevice);
    } else {
      // the REAL*8 IJACOBIAN in a buffer of its own, rounded into L.jacb
      double* d_j64 = nullptr;
      const size_t nj = (size_t)npix * np * nfreq;
      if ((rc = cuda_fail(cudaMalloc(&d_j64, nj * sizeof(double))))) break;
      rc = cuda_fail(cudaMemcpy(d_j64, jac64, nj * sizeof(double), cudaMemcpyHostToDevice));
      if (!rc) {
        k_f64_to_f32<<<(int)std::min<size_t>((nj + 255) / 256, (size_t)c->nsm * 16), 256, 0, c->stream>>>(
            nj, d_j64, L.jacb);
        rc = cuda_fail(cudaStreamSynchronize(c->stream));
      }
      cudaFree(d_j64);
      if (rc) break;
    }
    cudaMemcpy(L.diff, diff, (size_t)npix * nfreq * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(d_w, ones.data(), nfreq * sizeof(double), cudaMemcpyHostToDevice);
    if (big) {
      const int nb = (np + GT_M - 1) / GT_M;
      if ((rc = cuda_fail(cudaFuncSetAttribute(k_lm_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)GT_SMEM)))) break;
      k_lm_gram_tc<<<dim3(nb * (nb + 1) / 2, npix), 128, GT_SMEM, c->stream>>>(C, L, d_w, d_err);
      k_lm_grad<<<dim3((np + 7) / 8, npix), 256, 0, c->stream>>>(C, L, d_w);
      if (C.solver == 2)
        k_lm_cg_big<<<npix, 256, 6 * np * sizeof(double), c->stream>>>(C, L);
      else
        k_lm_svd_big<<<npix, 256, 2 * np * sizeof(double), c->stream>>>(C, L, d_svd);
    } else {
      k_lm_normal<<<(npix + 3) / 4, 128, 0, c->stream>>>(C, L, d_w);
      k_lm_solve<<<(npix + 3) / 4, 128, 0, c->stream>>>(C, L);
    }
    if ((rc = cuda_fail(cudaGetLastError()))) break;
    if ((rc = cuda_fail(cudaStreamSynchronize(c->stream)))) break;
    rc = cuda_fail(cudaMemcpy(delta, L.delta, (size_t)npix * np * sizeof(double), cudaMemcpyDeviceToHost));
    if (!rc && d_err) {
      int e = 0;
      rc = cuda_fail(cudaMemcpy(&e, d_err, sizeof(int), cudaMemcpyDeviceToHost));
      if (!rc && e) rc = FZ_ERR_CUDA;
    }
  } while (false);
  cudaFree(L.pix);
  cudaFree(L.skip);
  cudaFree(L.st);
  cudaFree(L.jacb);
  cudaFree(L.diff);
  cudaFree(L.H);
  cudaFree(L.g);
  cudaFree(L.delta);
  cudaFree(L.pen);
  cudaFree(L.hss);
  cudaFree(d_w);
  cudaFree(d_ones);
  cudaFree(d_err);
  cudaFree(d_svd);
  return rc;
}

int fz_warm_start_device(fz_ctx* c, fz_mlp* mlp, int npix, const double* d_obs, const float* d_norm,
                         const float* d_base, float* d_models, void* stream) {
  if (!c || !mlp || npix <= 0 || !d_obs || !d_norm || !d_base || !d_models) return FZ_ERR_ARG;
  if (c->rf.np <= 0) return FZ_ERR_STATE;
  const int nf = 4 * c->numw, np = c->rf.np;
  int nin = 0, nout = 0;
  if (int rc = fz_mlp_io(mlp, &nin, &nout)) return rc;
  if (nin != nf || nout != np) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  cudaStream_t s = (cudaStream_t)stream;
  const size_t ny = (size_t)npix * np;
  if (ny + np > c->wsy_len) {
    FZ_CK(cudaStreamSynchronize(s));
    cudaFree(c->d_wsy);
    c->d_wsy = nullptr;
    c->wsy_len = 0;
    FZ_CK(cudaMalloc(&c->d_wsy, (ny + np) * sizeof(float)));
    c->wsy_len = ny + np;
  }
  if (int rc = fz_mlp_forward_obs_device(mlp, npix, d_obs, d_norm, d_norm + nf, c->d_wsy, stream)) return rc;
  float* cb = c->d_wsy + ny;   // CONTRACT(base), np floats behind the network's outputs
  k_ws_contract<<<1, 32, 0, s>>>(c->nz, c->rf, c->d_coef, d_base, cb);
  k_ws_expand<<<npix, 128, np * sizeof(float), s>>>(npix, c->nz, c->rf, c->d_coef, c->d_wsy, d_norm + 2 * nf,
                                                    d_norm + 2 * nf + np, d_base, cb, d_models);
  return cuda_fail(cudaGetLastError());
}

int fz_invert_warm(fz_ctx* c, fz_mlp* mlp, const float* norm, const float* base, int npix, const double* obs,
                   const double* target_chi2, int hydrostatic, const fz_lm_opts* opts, float* model_out,
                   double* chi2, int* iters, double* syn_out, int* status) {
  if (!c || !mlp || !norm || !base || npix <= 0 || !obs || !model_out || !chi2 || !iters) return FZ_ERR_ARG;
  if (c->rf.np <= 0) return FZ_ERR_STATE;
  FZ_CK(cudaSetDevice(c->device));
  const size_t nf = 4 * (size_t)c->numw, nm = 13 * (size_t)c->nz;
  cudaStream_t s = c->stream;
  // the staging of fz_invert, grown on demand (a call with no pixels of its
  // own runs it at zero size first)
  if ((size_t)npix > c->inv.cap) {
    FZ_CK(cudaStreamSynchronize(s));
    const size_t n = npix;
    inv_free(c);
    int rc = 0;
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.obs, n * nf * sizeof(double)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.init, n * nm * sizeof(float)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.out, n * nm * sizeof(float)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.chi, n * sizeof(double)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.tgt, n * sizeof(double)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.it, n * sizeof(int)));
    if (!rc) rc = cuda_fail(cudaMalloc(&c->inv.st, n * sizeof(int)));
    if (rc) {
      inv_free(c);
      return rc;
    }
    c->inv.cap = n;
  }
  if (syn_out && !c->inv.syn) FZ_CK(cudaMalloc(&c->inv.syn, c->inv.cap * nf * sizeof(double)));
  if (syn_out) c->inv.has_syn = true;
  const size_t nnorm = 2 * nf + 2 * (size_t)c->rf.np + nm;   // normalisation, then the base model
  if (nnorm > c->wsnorm_len) {
    cudaFree(c->d_wsnorm);
    c->d_wsnorm = nullptr;
    c->wsnorm_len = 0;
    FZ_CK(cudaMalloc(&c->d_wsnorm, nnorm * sizeof(float)));
    c->wsnorm_len = nnorm;
  }
  const size_t nn = 2 * nf + 2 * (size_t)c->rf.np;
  FZ_CK(cudaMemcpyAsync(c->d_wsnorm, norm, nn * sizeof(float), cudaMemcpyHostToDevice, s));
  FZ_CK(cudaMemcpyAsync(c->d_wsnorm + nn, base, nm * sizeof(float), cudaMemcpyHostToDevice, s));
  FZ_CK(cudaMemcpyAsync(c->inv.obs, obs, npix * nf * sizeof(double), cudaMemcpyHostToDevice, s));
  if (target_chi2)
    FZ_CK(cudaMemcpyAsync(c->inv.tgt, target_chi2, npix * sizeof(double), cudaMemcpyHostToDevice, s));
  // the warm-start models straight into the inversion's initial models
  if (int rc = fz_warm_start_device(c, mlp, npix, c->inv.obs, c->d_wsnorm, c->d_wsnorm + nn, c->inv.init, s))
    return rc;
  fz_lm_opts o{};
  if (opts) o = *opts;
  if (opts && opts->fallback_model) {
    if (!c->inv.fb) FZ_CK(cudaMalloc(&c->inv.fb, nm * sizeof(float)));
    FZ_CK(cudaMemcpyAsync(c->inv.fb, opts->fallback_model, nm * sizeof(float), cudaMemcpyHostToDevice, s));
    o.fallback_model = c->inv.fb;
  }
  if (opts && opts->state_out) {
    if ((size_t)npix > c->inv.state_cap) {
      cudaFree(c->inv.state);
      c->inv.state = nullptr;
      c->inv.state_cap = 0;
      FZ_CK(cudaMalloc(&c->inv.state, (size_t)npix * 5 * sizeof(double)));
      c->inv.state_cap = npix;
    }
    o.state_out = c->inv.state;
  }
  int rc = fz_invert_device(c, npix, c->inv.obs, c->inv.init, target_chi2 ? c->inv.tgt : nullptr, hydrostatic,
                            opts ? &o : nullptr, c->inv.out, c->inv.chi, c->inv.it, syn_out ? c->inv.syn : nullptr,
                            c->inv.st, s);
  if (rc) return rc;
  FZ_CK(cudaMemcpyAsync(model_out, c->inv.out, npix * nm * sizeof(float), cudaMemcpyDeviceToHost, s));
  FZ_CK(cudaMemcpyAsync(chi2, c->inv.chi, npix * sizeof(double), cudaMemcpyDeviceToHost, s));
  FZ_CK(cudaMemcpyAsync(iters, c->inv.it, npix * sizeof(int), cudaMemcpyDeviceToHost, s));
  if (status) FZ_CK(cudaMemcpyAsync(status, c->inv.st, npix * sizeof(int), cudaMemcpyDeviceToHost, s));
  if (syn_out) FZ_CK(cudaMemcpyAsync(syn_out, c->inv.syn, npix * nf * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (opts && opts->state_out)
    FZ_CK(cudaMemcpyAsync(opts->state_out, c->inv.state, (size_t)npix * 5 * sizeof(double), cudaMemcpyDeviceToHost,
                          s));
  FZ_CK(cudaStreamSynchronize(s));
  return 0;
}

int fz_lm_perturbation(fz_ctx* c, int npix, int np, int nfreq, const double* jac, const double* diff,
                       const double* lambda, const double* reg_pen, const double* reg_hss, int dtype, double svdtol,
                       double* delta) {
  if (!jac) return FZ_ERR_ARG;
  return lm_perturbation_host(c, npix, np, nfreq, jac, nullptr, diff, lambda, reg_pen, reg_hss, dtype, svdtol, delta);
}

int fz_lm_perturbation_f32(fz_ctx* c, int npix, int np, int nfreq, const float* jac, const double* diff,
                           const double* lambda, const double* reg_pen, const double* reg_hss, int dtype,
                           double svdtol, double* delta) {
  if (!jac) return FZ_ERR_ARG;
  return lm_perturbation_host(c, npix, np, nfreq, nullptr, jac, diff, lambda, reg_pen, reg_hss, dtype, svdtol, delta);
}

int fz_lm_update_lambda_device(int n, const double* d_chicur, double* d_chipre, double* d_lambda, double* d_steps,
                               double* d_precyc, void* stream) {
  if (n <= 0 || !d_chicur || !d_chipre || !d_lambda || !d_steps || !d_precyc) return FZ_ERR_ARG;
  k_lm_lambda<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, d_chicur, d_chipre, d_lambda, d_steps, d_precyc);
  return cuda_fail(cudaGetLastError());
}

int fz_lm_update_lambda(int n, const double* chicur, double* chipre, double* lambda, double* steps, double* precyc) {
  if (n <= 0 || !chicur || !chipre || !lambda || !steps || !precyc) return FZ_ERR_ARG;
  double* d = nullptr;
  const size_t b = (size_t)n * sizeof(double);
  FZ_CK(cudaMalloc(&d, 5 * b));
  int rc = 0;
  const double* src[5] = {chicur, chipre, lambda, steps, precyc};
  for (int k = 0; k < 5 && !rc; ++k) rc = cuda_fail(cudaMemcpy(d + (size_t)k * n, src[k], b, cudaMemcpyHostToDevice));
  if (!rc) rc = fz_lm_update_lambda_device(n, d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n, d + 4 * (size_t)n, nullptr);
  double* dst[4] = {chipre, lambda, steps, precyc};
  for (int k = 0; k < 4 && !rc; ++k)
    rc = cuda_fail(cudaMemcpy(dst[k], d + (size_t)(k + 1) * n, b, cudaMemcpyDeviceToHost));
  cudaFree(d);
  return rc;
}

int fz_lm_rearange_device(fz_ctx* c, int npix, float* d_models, const double* d_delta, int node_expansion,
                          void* stream) {
  if (!c || npix <= 0 || !d_models || !d_delta || node_expansion < 0 || node_expansion > 2) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  fz_lm_opts o{};
  o.node_expansion = node_expansion;
  LMConf C;
  int rc = lm_conf(c, npix, &o, C);
  if (rc) return rc;
  LMSlots L{};
  L.S = npix;
  L.mcur = d_models;
  L.delta = const_cast<double*>(d_delta);
  const size_t usm = (size_t)(C.nz + 3 * C.np) * sizeof(double) + (size_t)C.nz * sizeof(float);
  k_lm_update<<<npix, 128, usm, (cudaStream_t)stream>>>(C, L, c->d_coef64);
  return cuda_fail(cudaGetLastError());
}

int fz_lm_rearange(fz_ctx* c, int npix, float* models, const double* delta, int node_expansion) {
  if (!c || npix <= 0 || !models || !delta) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  if (c->rf.np <= 0) return FZ_ERR_STATE;
  const size_t mb = (size_t)npix * 13 * c->nz * sizeof(float), db = (size_t)npix * c->rf.np * sizeof(double);
  float* dm = nullptr;
  double* dd = nullptr;
  int rc = cuda_fail(cudaMalloc(&dm, mb));
  if (!rc) rc = cuda_fail(cudaMalloc(&dd, db));
  if (!rc) rc = cuda_fail(cudaMemcpy(dm, models, mb, cudaMemcpyHostToDevice));
  if (!rc) rc = cuda_fail(cudaMemcpy(dd, delta, db, cudaMemcpyHostToDevice));
  if (!rc) rc = fz_lm_rearange_device(c, npix, dm, dd, node_expansion, c->stream);
  if (!rc) rc = cuda_fail(cudaStreamSynchronize(c->stream));
  if (!rc) rc = cuda_fail(cudaMemcpy(models, dm, mb, cudaMemcpyDeviceToHost));
  cudaFree(dm);
  cudaFree(dd);
  return rc;
}

int fz_rte_solve_device(int ncol, int nz, int nw, const float* d_eta, const float* d_src, const double* d_zz,
                        const int* d_bnd, double* d_out, void* stream) {
  if (ncol <= 0 || nz <= 1 || nw <= 0 || !d_eta || !d_src || !d_zz || !d_out) return FZ_ERR_ARG;
  const long long n = (long long)ncol * nw;
  k_rte<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(ncol, nz, nw, d_eta, d_src, d_zz, d_bnd,
                                                                          d_out);
  return cuda_fail(cudaGetLastError());
}

int fz_rte_solve(int ncol, int nz, int nw, const float* eta, const float* src, const double* zz, const int* bnd,
                 double* out) {
  if (ncol <= 0 || nz <= 1 || nw <= 0 || !eta || !src || !zz || !out) return FZ_ERR_ARG;
  const size_t ne = (size_t)ncol * nz * 7 * nw, ns = (size_t)ncol * nz * nw, no = (size_t)ncol * nw * 4;
  float *de = nullptr, *ds = nullptr;
  double *dz = nullptr, *dout = nullptr;
  int* db = nullptr;
  int rc = cuda_fail(cudaMalloc(&de, ne * sizeof(float)));
  if (!rc) rc = cuda_fail(cudaMalloc(&ds, ns * sizeof(float)));
  if (!rc) rc = cuda_fail(cudaMalloc(&dz, nz * sizeof(double)));
  if (!rc) rc = cuda_fail(cudaMalloc(&dout, no * sizeof(double)));
  if (!rc && bnd) rc = cuda_fail(cudaMalloc(&db, (size_t)ncol * nz * sizeof(int)));
  if (!rc) rc = cuda_fail(cudaMemcpy(de, eta, ne * sizeof(float), cudaMemcpyHostToDevice));
  if (!rc) rc = cuda_fail(cudaMemcpy(ds, src, ns * sizeof(float), cudaMemcpyHostToDevice));
  if (!rc) rc = cuda_fail(cudaMemcpy(dz, zz, nz * sizeof(double), cudaMemcpyHostToDevice));
  if (!rc && bnd) rc = cuda_fail(cudaMemcpy(db, bnd, (size_t)ncol * nz * sizeof(int), cudaMemcpyHostToDevice));
  if (!rc) rc = fz_rte_solve_device(ncol, nz, nw, de, ds, dz, db, dout, nullptr);
  if (!rc) rc = cuda_fail(cudaMemcpy(out, dout, no * sizeof(double), cudaMemcpyDeviceToHost));
  cudaFree(de);
  cudaFree(ds);
  cudaFree(dz);
  cudaFree(dout);
  cudaFree(db);
  return rc;
}

int fz_voigt(int n, const float* a, const float* v, float* h, float* f) {
  if (n <= 0 || !a || !v || !h || !f) return FZ_ERR_ARG;
  float* d = nullptr;
  const size_t b = (size_t)n * sizeof(float);
  FZ_CK(cudaMalloc(&d, 4 * b));
  int rc = cuda_fail(cudaMemcpy(d, a, b, cudaMemcpyHostToDevice));
  if (!rc) rc = cuda_fail(cudaMemcpy(d + n, v, b, cudaMemcpyHostToDevice));
  if (!rc) {
    k_voigt<<<(n + 255) / 256, 256>>>(n, d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n);
    rc = cuda_fail(cudaGetLastError());
  }
  if (!rc) rc = cuda_fail(cudaMemcpy(h, d + 2 * (size_t)n, b, cudaMemcpyDeviceToHost));
  if (!rc) rc = cuda_fail(cudaMemcpy(f, d + 3 * (size_t)n, b, cudaMemcpyDeviceToHost));
  cudaFree(d);
  return rc;
}

static int forward_rf_host(fz_ctx* c, int ncol, const float* model, int hydrostatic, double* syn, float* jac,
                           float* model_out, int* status, bool full) {
  if (!c || ncol <= 0 || !model || !syn || !jac) return FZ_ERR_ARG;
  if (!full && c->rf.np <= 0) return FZ_ERR_STATE;
  const int npj = full ? NSLOT * c->nz : c->rf.np;
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
  const size_t jb = (size_t)ncol * npj * 4 * c->numw * sizeof(float);
  if ((size_t)ncol * npj > c->jac_cols) {
    cudaFree(c->d_jac);
    c->d_jac = nullptr;
    c->jac_cols = 0;
    FZ_CK(cudaMalloc(&c->d_jac, jb));
    c->jac_cols = (size_t)ncol * npj;
  }
  cudaStream_t s = c->stream;
  const size_t mb = (size_t)ncol * 13 * c->nz * sizeof(float);
  FZ_CK(cudaMemcpyAsync(c->d_model, model, mb, cudaMemcpyHostToDevice, s));
  int rc = launch_forward_rf(c, ncol, c->d_model, hydrostatic, c->d_syn, c->d_jac, c->d_model, c->d_status, s, full);
  if (rc) return rc;
  FZ_CK(cudaMemcpyAsync(syn, c->d_syn, (size_t)ncol * 4 * c->numw * sizeof(double), cudaMemcpyDeviceToHost, s));
  FZ_CK(cudaMemcpyAsync(jac, c->d_jac, jb, cudaMemcpyDeviceToHost, s));
  if (model_out) FZ_CK(cudaMemcpyAsync(model_out, c->d_model, mb, cudaMemcpyDeviceToHost, s));
  if (status) FZ_CK(cudaMemcpyAsync(status, c->d_status, ncol * sizeof(int), cudaMemcpyDeviceToHost, s));
  FZ_CK(cudaStreamSynchronize(s));
  return 0;
}

int fz_forward_rf(fz_ctx* c, int ncol, const float* model, int hydrostatic, double* syn, float* jac, float* model_out,
                  int* status) {
  return forward_rf_host(c, ncol, model, hydrostatic, syn, jac, model_out, status, false);
}

int fz_forward_rf_full(fz_ctx* c, int ncol, const float* model, int hydrostatic, double* syn, float* rf,
                       float* model_out, int* status) {
  return forward_rf_host(c, ncol, model, hydrostatic, syn, rf, model_out, status, true);
}

int fz_forward_rf_full_device(fz_ctx* c, int ncol, const float* d_model, int hydrostatic, double* d_syn, float* d_rf,
                              float* d_model_out, int* d_status, void* stream) {
  if (!c || ncol <= 0 || !d_model || !d_syn || !d_rf || !d_model_out) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  return launch_forward_rf(c, ncol, d_model, hydrostatic, d_syn, d_rf, d_model_out, d_status, (cudaStream_t)stream,
                           true);
}

// ------------------------------------------------------------- autotuner
// Launch shapes of the RF path measured on the caller's columns: every
// candidate of a kernel runs once untimed and three times between CUDA events
// on the context's stream, with the inputs the previous kernel of the chain
// left (the kernels are deterministic, so repeated launches do the same
// work); the fastest is kept in the context.
int fz_autotune_forward(fz_ctx* c, int ncol, const float* d_model, int hydrostatic, fz_tune* out) {
  if (!c || ncol <= 0 || !d_model) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  int rc = ensure_rf_scratch(c, ncol);
  if (rc) return rc;
  cudaStream_t s = c->stream;
  float* d_mout = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  struct Cleanup {
    float*& m;
    cudaEvent_t &a, &b;
    ~Cleanup() {
      cudaFree(m);
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } cl{d_mout, e0, e1};
  FZ_CK(cudaMalloc(&d_mout, (size_t)ncol * 13 * c->nz * sizeof(float)));
  FZ_CK(cudaEventCreate(&e0));
  FZ_CK(cudaEventCreate(&e1));
  auto timed = [&](auto&& launch, float& ms) -> int {
    launch();
    FZ_CK(cudaEventRecord(e0, s));
    for (int r = 0; r < 3; ++r) launch();
    FZ_CK(cudaEventRecord(e1, s));
    FZ_CK(cudaEventSynchronize(e1));
    FZ_CK(cudaGetLastError());
    FZ_CK(cudaEventElapsedTime(&ms, e0, e1));
    ms /= 3.0f;
    return 0;
  };
  float best = 0.0f, ms = 0.0f, tchain = 0.0f, tchem = 0.0f, topac = 0.0f;
  int bw = c->tune.chain_warps, bl = c->tune.chain_lanes;
  // lanes per column stay automatic (by batch size: the inversion's batches
  // shrink from the full pool to a few columns, so one fixed value measured
  // on this batch would not fit them)
  static const int kWarps[] = {1, 2, 4};
  static const int kLanes[] = {0};
  for (int i = 0; i < 3; ++i) {
    const int w = kWarps[i % 3], l = kLanes[i / 3];
    if ((rc = timed([&] { launch_chain(c, ncol, d_model, d_mout, nullptr, hydrostatic, w, s, l); }, ms))) return rc;
    if (i == 0 || ms < best) best = ms, bw = w, bl = l;
  }
  tchain = best;
  launch_chain(c, ncol, d_model, d_mout, nullptr, hydrostatic, bw, s, bl);
  int bb = c->tune.chemder_bpsm;
  static const int kBpsm[] = {8, 16, 32, 64, 0};
  for (int i = 0; i < 5; ++i) {
    const int b = kBpsm[i];
    if ((rc = timed([&] { launch_chemder(c, ncol, d_mout, b, s); }, ms))) return rc;
    if (i == 0 || ms < best) best = ms, bb = b;
  }
  tchem = best;
  int bt = c->tune.opacrf_threads;
  static const int kThreads[] = {64, 128, 256};
  for (int i = 0; i < 3; ++i) {
    const int t = kThreads[i];
    if ((rc = timed([&] { launch_opac_rf(c, ncol, d_mout, t, s); }, ms))) return rc;
    if (i == 0 || ms < best) best = ms, bt = t;
  }
  topac = best;
  c->tune.chain_warps = bw;
  c->tune.chain_lanes = bl;
  c->tune.chemder_bpsm = bb;
  c->tune.opacrf_threads = bt;
  if (out) {
    out->chain_warps = bw;
    out->chain_lanes = bl;
    out->chemder_blocks_per_sm = bb;
    out->opac_rf_threads = bt;
    out->lm_slots = c->tune.lm_slots;
    out->chain_ms = tchain;
    out->chemder_ms = tchem;
    out->opac_rf_ms = topac;
  }
  return 0;
}

// Pixels in flight of the batched inversion: each candidate inverts the same
// npix pixels (device buffers as fz_invert_device) and the highest
// pixels/s is kept as the default of fz_lm_opts.slots == 0.
int fz_autotune_lm(fz_ctx* c, int npix, const double* d_obs, const float* d_init, const double* d_target_chi2,
                   int hydrostatic, const fz_lm_opts* opts, const int* candidates, int ncand, fz_tune* out) {
  if (!c || npix <= 0 || !d_obs || !d_init || !candidates || ncand <= 0) return FZ_ERR_ARG;
  FZ_CK(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  float* d_mo = nullptr;
  double* d_chi = nullptr;
  int* d_it = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = 0;
  float bestrate = -1.0f;
  int bests = c->tune.lm_slots;
  do {
    if ((rc = cuda_fail(cudaMalloc(&d_mo, (size_t)npix * 13 * c->nz * sizeof(float))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_chi, (size_t)npix * sizeof(double))))) break;
    if ((rc = cuda_fail(cudaMalloc(&d_it, (size_t)npix * sizeof(int))))) break;
    if ((rc = cuda_fail(cudaEventCreate(&e0)))) break;
    if ((rc = cuda_fail(cudaEventCreate(&e1)))) break;
    fz_lm_opts o{};
    if (opts) o = *opts;
    for (int i = 0; i < ncand && !rc; ++i) {
      if (candidates[i] <= 0) {
        rc = FZ_ERR_ARG;
        break;
      }
      o.slots = std::min(candidates[i], npix);
      if ((rc = cuda_fail(cudaEventRecord(e0, s)))) break;
      if ((rc = fz_invert_device(c, npix, d_obs, d_init, d_target_chi2, hydrostatic, &o, d_mo, d_chi, d_it, nullptr,
                                 nullptr, s)))
        break;
      if ((rc = cuda_fail(cudaEventRecord(e1, s)))) break;
      if ((rc = cuda_fail(cudaEventSynchronize(e1)))) break;
      float ms = 0.0f;
      if ((rc = cuda_fail(cudaEventElapsedTime(&ms, e0, e1)))) break;
      const float rate = (float)npix / (ms * 1e-3f);
      if (rate > bestrate) bestrate = rate, bests = o.slots;
    }
  } while (false);
  cudaFree(d_mo);
  cudaFree(d_chi);
  cudaFree(d_it);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (rc) return rc;
  c->tune.lm_slots = bests;
  if (out) {
    out->lm_slots = bests;
    out->lm_pixels_per_s = bestrate;
  }
  return 0;
}

int fz_tune_get(fz_ctx* c, fz_tune* t) {
  if (!c || !t) return FZ_ERR_ARG;
  t->chain_warps = c->tune.chain_warps;
  t->chain_lanes = c->tune.chain_lanes;
  t->chemder_blocks_per_sm = c->tune.chemder_bpsm;
  t->opac_rf_threads = c->tune.opacrf_threads;
  t->lm_slots = c->tune.lm_slots;
  return 0;
}

int fz_tune_set(fz_ctx* c, const fz_tune* t) {
  if (!c || !t) return FZ_ERR_ARG;
  if (t->chain_warps < 1 || t->chain_warps > 4 || (t->chain_lanes != 0 && t->chain_lanes != 32 && t->chain_lanes != 16) ||
      t->chemder_blocks_per_sm < 0 || t->lm_slots < 1 ||
      (t->opac_rf_threads != 64 && t->opac_rf_threads != 128 && t->opac_rf_threads != 256))
    return FZ_ERR_ARG;
  c->tune.chain_warps = t->chain_warps;
  c->tune.chain_lanes = t->chain_lanes;
  c->tune.chemder_bpsm = t->chemder_blocks_per_sm;
  c->tune.opacrf_threads = t->opac_rf_threads;
  c->tune.lm_slots = t->lm_slots;
  return 0;
}

}  // extern "C"

// ------------------------------------------------ allocation-free variant
// Scratch of fz_forward_device_static: one file-scope device array, shared
// by every call on a device and kept for the life of the process.  It holds
// the per-height (nH, ne) pairs and the opacity slab of one batch of columns.
#define FZ_NOALLOC_SCRATCH_BYTES (64ull << 20)
static __device__ __align__(256) unsigned char g_fz_noalloc_scratch[FZ_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device` (the current device).  In
// host code the array's name is only a host-side stand-in, so the address is
// looked up once per device with cudaGetSymbolAddress.
int noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return FZ_ERR_ARG;
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_fz_noalloc_scratch);
    if (e != cudaSuccess) {
      std::fprintf(stderr, "fz_b200: cudaGetSymbolAddress of the static scratch failed: %s\n", cudaGetErrorString(e));
      return FZ_ERR_CUDA;
    }
    g_noalloc_ptr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[device]);
  return 0;
}
}  // namespace

extern "C" {

int fz_forward_device_static(fz_ctx* c, int ncol, const float* d_model, int hydrostatic, double* d_syn,
                             float* d_model_out, int* d_status, void* stream) {
  if (!c || ncol <= 0 || !d_model || !d_syn || !d_model_out) return FZ_ERR_ARG;
  if (hydrostatic < 0 || hydrostatic > 2) return FZ_ERR_ARG;
  const size_t chem_bytes = ((size_t)ncol * c->nz * sizeof(double2) + 255) & ~(size_t)255;
  const size_t slab_bytes = (size_t)ncol * c->nz * c->sw * sizeof(float);
  if (chem_bytes + slab_bytes > FZ_NOALLOC_SCRATCH_BYTES) {
    std::fprintf(stderr,
                 "fz_b200: fz_forward_device_static: %d columns x %d heights need %zu bytes of scratch, "
                 "more than the %llu-byte static array; split the batch\n",
                 ncol, c->nz, chem_bytes + slab_bytes, (unsigned long long)FZ_NOALLOC_SCRATCH_BYTES);
    return FZ_ERR_LIMIT;
  }
  FZ_CK(cudaSetDevice(c->device));
  unsigned char* base = nullptr;
  const int rc = noalloc_scratch(c->device, &base);
  if (rc) return rc;
  double2* chem = reinterpret_cast<double2*>(base);
  float* slab = reinterpret_cast<float*>(base + chem_bytes);
  cudaStream_t s = (cudaStream_t)stream;
  // Every scratch word a kernel reads is written earlier in the same call
  // (k_chain fills chem, k_opac fills the slab rows), so nothing is cleared.
  if (d_status) FZ_CK(cudaMemsetAsync(d_status, 0, ncol * sizeof(int), s));
  // the chemistry chain with the context's launch shape (tuned or default),
  // so that both entry points run the same schedule and agree bit for bit
  launch_k_chain(c, ncol, d_model, d_model_out, d_status, hydrostatic, c->tune.chain_warps, c->tune.chain_lanes, s,
                 chem, nullptr, nullptr, false);
  FZ_CK(cudaGetLastError());
  const size_t total = (size_t)ncol * c->nz;
  const int blocks = (int)std::min<size_t>((total + 255) / 256, (size_t)c->nsm * 16);
  k_opac<<<blocks, 256, 0, s>>>(c->d_params, c->d_consts, ncol, d_model_out, chem, slab);
  FZ_CK(cudaGetLastError());
  const int threads = (c->numw + 31) & ~31;
  const size_t sms = (size_t)c->nz * c->sw * sizeof(float);
  k_synth<<<ncol, threads, sms, s>>>(c->d_params, c->d_lam, c->d_gain, ncol, slab, d_syn, d_model_out, d_status);
  FZ_CK(cudaGetLastError());
  return launch_lsf<double>(c, d_syn, (long long)ncol * 4, 4, s);   // allocates nothing
}

int fz_forward(fz_ctx* c, int ncol, const float* model, int hydrostatic, double* syn, float* model_out,
               int* status) {
  if (!c || ncol <= 0 || !model || !syn) return FZ_ERR_ARG;
  if (hydrostatic < 0 || hydrostatic > 2) return FZ_ERR_ARG;
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
