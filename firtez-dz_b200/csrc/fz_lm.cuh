// Batched pixel-wise Levenberg-Marquardt (sm_100a), included by fz_cuda.cu.
//
// One inversion = a pool of S slots, each holding one pixel: its observed
// Stokes vector, current and best model, synthesis and node Jacobian, and the
// LM state of the reference (INV_SLA(1:9), src/invert3d.f90:275-286).  Every
// iteration runs, on all slots:
//   forward synthesis + node Jacobian of the current models (k_chain,
//   k_opac_rf, k_synth_rf);
//   k_lm_accept   chi2, accept/revert, lambda update (NEW_CALCULATE_CHI2,
//                 UPDATE_LAMBDA, src/get_dmodel.f90:917-1032), the weighted
//                 residual, the per-pixel stop rule (optionally a per-pixel
//                 chi2 goal); a finished pixel writes
//                 its best model out and its slot takes the next pixel of
//                 the work queue (a device counter);
//   k_lm_normal   H = Jn^T Jn on the tensor cores (mma.sync bf16, the FP32
//                 Jacobian split in hi + lo bf16 parts, hi*hi + hi*lo + lo*hi
//                 accumulated in FP32) and g = Jn^T r in FP64, Jn the
//                 normalised Jacobian of NORMALIZE_JACOB (:725-770);
//   k_lm_solve    one warp per pixel, FP64: (H + lambda diag H)^+ g by a
//                 one-sided Jacobi SVD with the reference's relative cut
//                 (GET_PERTURBATION/GET_INVERSE, src/lm.f90:61-204);
//   k_lm_update   REARANGE_DA_MODEL / SORT_DELTA_TO_ATMOSPHERE
//                 (:1715-2016): node clipping, SIR-like expansion, limits,
//                 the log tau5 taper of T.
#pragma once

namespace {

constexpr int LM_MAXNP = 16;    // the warp kernels' tile (mma.sync normal equations, warp SVD)
constexpr int LM_MAXNP_BIG = 1024;   // larger layouts: tcgen05 normal equations, CTA solvers
constexpr int LM_PAD = -1;      // empty slot
constexpr int LM_SKIP = 1;      // slot refilled this iteration: no step yet

struct LMConf {
  int np, nfreq, nz, npix;
  int maxsteps, maxit;
  double dchi2, svdtol, inu;
  double fallback;             // restart factor on the chi2 goal (0 = off)
  const float* fb_model;       // MODEL(NZ,13) a restarted pixel starts from
  int fb_steps;                // restart once STEPS reaches this while above fallback x goal
  int fb_free;                 // a restarted search ignores the goal
  int solver;                  // SOLVER_METHOD: 1 SVD (GET_INVERSE), 2 CG (NEW_CALCULATE_DELTA_UBICGSTAB)
  int node_exp;                // NODE_EXPANSION: 1 SIR/NICOLE-like, 2 STiC-like
  int reg;                     // vertical regularisation on (GET_IT_PENALTIES)
  double reg_hss[LM_MAXNP * LM_MAXNP];   // PEN_HSS = L^T L (model independent)
  int global_stop;             // MAKE_DECISION's field rule on the mean STEPS (steps summed in the queue)
  double* state_out;           // (npix, 5) final STEPS, chi2 cur, chi2 best, PRECYC, lambda; may be null
  int nodes_ref[8];            // node count per reference parameter
  int row_of[LM_MAXNP];        // model row of each node's parameter
  int par_of[LM_MAXNP];        // reference parameter (1-based) of each node
  double norm[LM_MAXNP];       // PARAM_NORMS of each node's parameter
  // np > LM_MAXNP: the same per-node tables in device memory
  const int* d_row;            // (np)
  const double* d_norm;        // (np)
  const double* d_hss;         // (np, np) PEN_HSS, when reg
};

__device__ __forceinline__ int lm_row(const LMConf& C, int j) { return C.np <= LM_MAXNP ? C.row_of[j] : C.d_row[j]; }
__device__ __forceinline__ double lm_nrm(const LMConf& C, int j) {
  return C.np <= LM_MAXNP ? C.norm[j] : C.d_norm[j];
}
__device__ __forceinline__ double lm_hss(const LMConf& C, int j, int i) {
  return C.np <= LM_MAXNP ? C.reg_hss[j * C.np + i] : C.d_hss[(size_t)j * C.np + i];
}

// Slot pool (device pointers), one allocation per field.
struct LMSlots {
  int S;
  int* pix;          // pixel index, LM_PAD if empty
  int* skip;         // LM_SKIP if the slot was refilled or restarted in this iteration or has no accepted model yet
  int* restarted;    // 0, or 1 + the first attempt's iterations once the pixel restarted from the fallback model
  int* iter;
  double* st;        // 5 per slot: chicur, chibest, lambda, steps, precyc
  float* mcur;       // (S, 13, nz)
  float* mbest;
  double* syn;       // (S, nfreq) forward output of mcur
  double* synb;      // best synthesis
  float* jacb;       // best Jacobian (S, np, nfreq), written by the RF pass of accepted models
  int* need_rf;      // 1 if the slot's model was accepted and the pixel goes on: its Jacobian is needed
  double* pen;       // PEN_RES of the best model (S, np), subtracted from J^T r; may be null
  double* hss;       // per-slot PEN_HSS (S, np, np) added to J^T J; null: C.reg_hss when C.reg
  int* rf_list;      // slots needing the RF pass, compacted (k_lm_rflist)
  double* obs;       // (S, nfreq)
  double* diff;      // weighted residual (S, nfreq)
  double* H;         // (S, np, np)
  double* g;         // (S, np)
  double* delta;     // (S, np)
  int* status;       // forward status (S)
};

struct LMQueue {
  int next;          // next pixel to load
  int done;          // finished pixels
  int active;        // occupied slots (k_lm_scan)
  int rf_count;      // slots in the RF pass of this iteration (k_lm_rflist)
  unsigned long long steps_sum;   // sum over the call's pixels of STEPS (global stop rule; two's complement)
  int tc_err;        // a tensor-core kernel gave up waiting (bounded mbarrier waits)
  int iters;         // iterations of the device-driven loop (k_lm_ctl)
  int gstop;         // the device-driven loop ended on the field-wide stop rule
  int pad;
};

// UPDATE_LAMBDA (src/get_dmodel.f90:917-956) with FACTOR = 0.01: an
// improvement moves the best chi2 to chicur and divides lambda by sqrt(10),
// lowering STEPS by one when it gains more than 1 % (else raising it); no
// improvement multiplies lambda by 3 right after a cycle start (PRECYC ~ 1,
// which it clears) or else by 10, and raises STEPS; lambda >= 1e-2.
__device__ __forceinline__ void lm_update_lambda(double chicur, double& chipre, double& lam, double& steps,
                                                 double& precyc) {
  const double gain = chipre - chicur;
  if (gain > 0) {
    steps = (gain > 0.01 * chipre) ? fmax(0.0, steps - 1.0) : steps + 1.0;
    chipre = chicur;
    lam = lam / sqrt(10.0);
  } else {
    if (fabs(precyc - 1.0) < 1.0e-2) {
      precyc = 0.0;
      lam = lam * 3.0;
    } else {
      lam = lam * 10.0;
    }
    steps = steps + 1.0;
  }
  lam = fmax(1.0e-2, lam);
}

// Batched UPDATE_LAMBDA on arrays (one thread per pixel).
__global__ void k_lm_lambda(int n, const double* __restrict__ chicur, double* __restrict__ chipre,
                            double* __restrict__ lam, double* __restrict__ steps, double* __restrict__ precyc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double cp = chipre[i], l = lam[i], st = steps[i], pc = precyc[i];
  lm_update_lambda(chicur[i], cp, l, st, pc);
  chipre[i] = cp;
  lam[i] = l;
  steps[i] = st;
  precyc[i] = pc;
}

// Final LM state of pixel p: INV_SLA(1:4) and INV_SLA(9) (STEPS, chi2 of the
// last model, best chi2, PRECYC, lambda; src/invert3d.f90:275-286).
__device__ __forceinline__ void lm_state_out(const LMConf& C, const double* st, int p) {
  if (!C.state_out) return;
  double* o = C.state_out + 5 * (size_t)p;
  o[0] = st[3];
  o[1] = st[0];
  o[2] = st[1];
  o[3] = st[4];
  o[4] = st[2];
}

// PARAM_NORMS (src/get_dmodel.f90:31), LOWLIM/UPPLIM (:1885-1901)
__constant__ double c_lm_norm[8] = {6000.0, 1.0e5, 1.0e-5, 1.0e3, 1.0e3, 1.0e3, 1.0e6, 6.0e2};
__constant__ double c_lm_low[8] = {2500.0, 1.0e-2, 1.0e-10, -5.0e4, -5.0e4, -5.0e4, -1.0e7, 1.0e-8};
__constant__ double c_lm_upp[8] = {1.8e4, 1.0e12, 1.0e10, 5.0e4, 5.0e4, 5.0e4, 1.0e7, 1.0e12};

// Node values of the free parameters of model m (13, nz): CONTRACT_VECTOR
// (src/get_dmodel.f90:861-880) over the hat table coef (nz, np), divided by
// PARAM_NORM -- the x of GET_IT_PENALTIES (:1041-1197).  Thread j < np.
__device__ __forceinline__ double lm_node_value(const LMConf& C, const float* __restrict__ m,
                                                const double* __restrict__ coef, int j) {
  const float* row = m + (size_t)lm_row(C, j) * C.nz;
  double a = 0.0, cs = 0.0;
  for (int k = 0; k < C.nz; ++k) {
    const double c = coef[(size_t)k * C.np + j];
    a += (double)row[k] * c;
    cs += c;
  }
  return a / cs / lm_nrm(C, j);
}

// PEN_RES_j = (PEN_HSS x)_j of model m for node j (x in shared xs)
__device__ __forceinline__ double lm_pen_res(const LMConf& C, const double* xs, int j) {
  double r = 0.0;
  for (int i = 0; i < C.np; ++i) r += lm_hss(C, j, i) * xs[i];
  return r;
}

__device__ __forceinline__ double block_sum_d(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < nw; ++i) s += red[i];
  return s;
}

// Load pixel p (or mark the slot empty) -- INITIALIZE_CYCLE's per-pixel state.
__device__ void lm_load_slot(const LMConf& C, const LMSlots& Sl, int s, int p, const double* __restrict__ obs_all,
                             const float* __restrict__ init_all) {
  const int nm = 13 * C.nz;
  if (p < C.npix) {
    // the best model starts as the initial one (INITIALIZE_CYCLE)
    for (int i = threadIdx.x; i < nm; i += blockDim.x) {
      const float v = init_all[(size_t)p * nm + i];
      Sl.mcur[(size_t)s * nm + i] = v;
      Sl.mbest[(size_t)s * nm + i] = v;
    }
    for (int i = threadIdx.x; i < C.nfreq; i += blockDim.x)
      Sl.obs[(size_t)s * C.nfreq + i] = obs_all[(size_t)p * C.nfreq + i];
    if (threadIdx.x == 0) {
      Sl.pix[s] = p;
      Sl.iter[s] = 0;
      Sl.restarted[s] = 0;
      double* st = Sl.st + 5 * (size_t)s;
      st[0] = 1.0e29;
      st[1] = 1.0e29;
      st[2] = 10.0;
      st[3] = 0.0;
      st[4] = 0.0;
    }
  } else if (threadIdx.x == 0) {
    Sl.pix[s] = LM_PAD;
  }
}

// One CTA per slot: initial fill from the queue.
__global__ void k_lm_fill(LMConf C, LMSlots Sl, LMQueue* q, const double* __restrict__ obs_all,
                          const float* __restrict__ init_all) {
  __shared__ int p;
  if (threadIdx.x == 0) p = atomicAdd(&q->next, 1);
  __syncthreads();
  lm_load_slot(C, Sl, blockIdx.x, p, obs_all, init_all);
  if (threadIdx.x == 0) Sl.skip[blockIdx.x] = 0;
}

// One CTA per slot: chi2, accept/revert, lambda, residual, stop rule, refill.
// The synthesis of the slot's model comes from the plain forward pass; the
// response functions are computed afterwards only where they are used: for
// an accepted model of a pixel that goes on (need_rf).  A rejected trial
// keeps the best model's Jacobian and a finished pixel needs none, as in
// the reference, which discards the response functions of rejected models
// (EQVDSYN keeps the best, src/get_dmodel.f90:995-1005).
__global__ void __launch_bounds__(256) k_lm_accept(LMConf C, LMSlots Sl, LMQueue* q, const double* __restrict__ w,
                                                   const double* __restrict__ obs_all,
                                                   const float* __restrict__ init_all,
                                                   const double* __restrict__ target, float* __restrict__ out_model,
                                                   double* __restrict__ out_chi, int* __restrict__ out_iter,
                                                   double* __restrict__ out_syn, int* __restrict__ out_status,
                                                   const double* __restrict__ coef) {
  __shared__ double red[8];
  extern __shared__ double sm_acc[];   // with regularisation: xs, pr (np each)
  double* xs = sm_acc;
  double* pr = sm_acc + C.np;
  __shared__ int acc, fin, early, np_next;
  const int s = blockIdx.x;
  if (threadIdx.x == 0) {
    Sl.skip[s] = 0;
    Sl.need_rf[s] = 0;
  }
  const int p = Sl.pix[s];
  if (p < 0) return;
  const int nf = C.nfreq, nm = 13 * C.nz;
  const double* obs = Sl.obs + (size_t)s * nf;
  const double* syn = Sl.syn + (size_t)s * nf;
  double e = 0.0;
  for (int i = threadIdx.x; i < nf; i += blockDim.x) {
    const double d = obs[i] - syn[i];
    e += d * d * w[i];
  }
  double chi = block_sum_d(e, red) / C.inu;
  if (C.reg) {
    // NEW_CALCULATE_CHI2 with regularisation (src/get_dmodel.f90:966-983):
    // + sum(PEN_RES^2) of the current model, PEN_FACTOR = 1
    const float* mc = Sl.mcur + (size_t)s * nm;
    for (int j = threadIdx.x; j < C.np; j += blockDim.x) xs[j] = lm_node_value(C, mc, coef, j);
    __syncthreads();
    for (int j = threadIdx.x; j < C.np; j += blockDim.x) pr[j] = lm_pen_res(C, xs, j);
    __syncthreads();
    double pp = 0.0;
    for (int j = 0; j < C.np; ++j) pp += pr[j] * pr[j];
    chi += pp;
  }
  double* st = Sl.st + 5 * (size_t)s;
  if (threadIdx.x == 0) {
    const double chibest = st[1];
    const int ok = Sl.status[s] == 0 && chi == chi;
    acc = ok && chi < chibest;
    double lam = st[2], steps = st[3], precyc = st[4], chipre = chibest;
    const double cc = ok ? chi : 1.0e300;
    lm_update_lambda(cc, chipre, lam, steps, precyc);
    if (C.global_stop)
      atomicAdd(&q->steps_sum, (unsigned long long)((long long)steps - (long long)st[3]));
    const int it = Sl.iter[s] + 1;
    Sl.iter[s] = it;
    // stop rule: steps > MAXSTEPS (GET_DMODEL3DS, src/get_dmodel.f90:1476),
    // the iteration cap, and an accepted step that improved chi2 by less than
    // dchi2 (relative)
    const bool small = acc && chibest < 1.0e29 && (chibest - cc) < C.dchi2 * chibest;
    // optional per-pixel goal: stop once the best chi2 reaches it
    const bool goal = target != nullptr && !(C.fb_free && Sl.restarted[s]) && chipre <= target[p];
    fin = steps > (double)C.maxsteps || it >= C.maxit || small || goal;
    // an early restart: the search has stagnated fb_steps times and is still
    // above fallback x its goal
    early = !fin && C.fallback > 0.0 && C.fb_model && target && !Sl.restarted[s] && steps >= (double)C.fb_steps &&
            chipre > C.fallback * target[p];
    st[0] = chi;
    st[1] = chipre;
    st[2] = lam;
    st[3] = steps;
    st[4] = precyc;
  }
  __syncthreads();
  if (acc) {
    const float* mc = Sl.mcur + (size_t)s * nm;
    float* mb = Sl.mbest + (size_t)s * nm;
    for (int i = threadIdx.x; i < nm; i += blockDim.x) mb[i] = mc[i];
    double* sb = Sl.synb + (size_t)s * nf;
    for (int i = threadIdx.x; i < nf; i += blockDim.x) sb[i] = syn[i];
    if (threadIdx.x == 0 && !fin && !early) Sl.need_rf[s] = 1;
  } else {
    const float* mb = Sl.mbest + (size_t)s * nm;
    float* mc = Sl.mcur + (size_t)s * nm;
    for (int i = threadIdx.x; i < nm; i += blockDim.x) mc[i] = mb[i];
  }
  __syncthreads();
  if (C.reg && Sl.pen && !fin) {
    // GET_IT_PENALTIES of the best model for the normal equations: after an
    // accepted step the current one, after a rejection the restored one
    // (:1010-1015)
    if (!acc) {
      const float* mb = Sl.mbest + (size_t)s * nm;
      for (int j = threadIdx.x; j < C.np; j += blockDim.x) xs[j] = lm_node_value(C, mb, coef, j);
      __syncthreads();
      for (int j = threadIdx.x; j < C.np; j += blockDim.x) pr[j] = lm_pen_res(C, xs, j);
      __syncthreads();
    }
    for (int j = threadIdx.x; j < C.np; j += blockDim.x) Sl.pen[(size_t)s * C.np + j] = pr[j];
  }
  if ((fin || early) && C.fallback > 0.0 && C.fb_model && target && !Sl.restarted[s] &&
      st[1] > C.fallback * target[p]) {
    // the search ended above fallback x its goal: start once more from the
    // fallback model (INITIALIZE_CYCLE's state), the goal kept
    float* mc = Sl.mcur + (size_t)s * nm;
    float* mb = Sl.mbest + (size_t)s * nm;
    for (int i = threadIdx.x; i < nm; i += blockDim.x) mc[i] = mb[i] = C.fb_model[i];
    if (threadIdx.x == 0) {
      if (C.global_stop) atomicAdd(&q->steps_sum, (unsigned long long)(-(long long)st[3]));
      st[0] = 1.0e29;
      st[1] = 1.0e29;
      st[2] = 10.0;
      st[3] = 0.0;
      st[4] = 0.0;
      Sl.restarted[s] = 1 + Sl.iter[s];
      Sl.iter[s] = 0;
      Sl.skip[s] = LM_SKIP;
    }
    return;
  }
  if (fin) {
    // the pixel's result is its best model (END_CYCLE, src/invert3d.f90:306-312)
    const float* mb = Sl.mbest + (size_t)s * nm;
    for (int i = threadIdx.x; i < nm; i += blockDim.x) out_model[(size_t)p * nm + i] = mb[i];
    if (out_syn)
      for (int i = threadIdx.x; i < nf; i += blockDim.x) out_syn[(size_t)p * nf + i] = Sl.synb[(size_t)s * nf + i];
    if (threadIdx.x == 0) {
      out_chi[p] = st[1];
      out_iter[p] = Sl.iter[s] + (Sl.restarted[s] > 0 ? Sl.restarted[s] - 1 : 0);
      if (out_status) out_status[p] = st[1] < 1.0e29 ? 0 : FZ_NAN;
      lm_state_out(C, st, p);
      atomicAdd(&q->done, 1);
      np_next = atomicAdd(&q->next, 1);
      Sl.skip[s] = LM_SKIP;
    }
    __syncthreads();
    lm_load_slot(C, Sl, s, np_next, obs_all, init_all);
    return;
  }
  if (st[1] >= 1.0e29) {
    // no model of this attempt has been accepted yet (its first synthesis
    // failed): there is no Jacobian to step from, so the initial model is
    // tried again, each failure raising STEPS until the stop rule ends the
    // pixel with its initial model and a non-zero status
    if (threadIdx.x == 0) Sl.skip[s] = LM_SKIP;
    return;
  }
  // weighted residual of the best synthesis (:1027)
  const double* sb = Sl.synb + (size_t)s * nf;
  double* df = Sl.diff + (size_t)s * nf;
  const double rin = 1.0 / sqrt(C.inu);
  for (int i = threadIdx.x; i < nf; i += blockDim.x) df[i] = (obs[i] - sb[i]) * sqrt(w[i]) * rin;
}

// bf16 split of a float: hi = RN(x), lo = RN(x - hi)
__device__ __forceinline__ void bf16_split(float x, unsigned short& hi, unsigned short& lo) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
  hi = __bfloat16_as_ushort(h);
  lo = __bfloat16_as_ushort(l);
}

__device__ __forceinline__ unsigned pack2(unsigned short a, unsigned short b) {
  return (unsigned)a | ((unsigned)b << 16);
}

__device__ __forceinline__ void mma_bf16(float c[4], const unsigned a[4], const unsigned b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One warp per slot: H = Jn^T Jn (np <= 16) on the tensor cores and
// g = Jn^T r in FP64.  Jn(r, c) = J(r, c) sqrt(w_r / INU) PARAM_NORM(c).
// Per k-step of 16 frequencies a thread holds rows {grp, grp+8} x
// frequencies {2t, 2t+1, 2t+8, 2t+9} of Jn^T: exactly its A fragment, and
// (column grp of tile 0, column grp+8 of tile 1) its B fragments.
// With list, warp i serves slot list[i] for i < *nlist: the inversion passes
// the accepted slots (rf_list).  H and g depend only on the best model's
// Jacobian, synthesis and penalties, which change only on an accepted step;
// a rejected trial leaves them as the last accepted step computed them, bit
// for bit, and k_lm_solve reads them again with the new lambda.
__global__ void __launch_bounds__(128) k_lm_normal(LMConf C, LMSlots Sl, const double* __restrict__ w,
                                                   const int* __restrict__ list = nullptr,
                                                   const int* __restrict__ nlist = nullptr) {
  const int lane = threadIdx.x & 31;
  int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (list) {
    if (s >= *nlist) return;
    s = list[s];
  }
  if (s >= Sl.S) return;
  if (Sl.pix[s] < 0 || Sl.skip[s]) return;
  const int nf = C.nfreq, np = C.np;
  const float* J = Sl.jacb + (size_t)s * np * nf;
  const int grp = lane >> 2, t = lane & 3;
  const int m0 = grp, m1 = grp + 8;
  const float n0 = m0 < np ? (float)C.norm[m0] : 0.0f, n1 = m1 < np ? (float)C.norm[m1] : 0.0f;
  const float* r0 = J + (size_t)(m0 < np ? m0 : 0) * nf;
  const float* r1 = J + (size_t)(m1 < np ? m1 : 0) * nf;
  const float rin = (float)(1.0 / sqrt(C.inu));
  float c0[4] = {0, 0, 0, 0}, c1[4] = {0, 0, 0, 0};
  for (int k0 = 0; k0 < nf; k0 += 16) {
    float v[2][4];   // [row m0/m1][freq 2t, 2t+1, 2t+8, 2t+9]
    const int ks[4] = {k0 + 2 * t, k0 + 2 * t + 1, k0 + 2 * t + 8, k0 + 2 * t + 9};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const bool in = ks[i] < nf;
      const float sw = in ? sqrtf((float)w[ks[i]]) * rin : 0.0f;
      v[0][i] = (in && m0 < np) ? r0[ks[i]] * sw * n0 : 0.0f;
      v[1][i] = (in && m1 < np) ? r1[ks[i]] * sw * n1 : 0.0f;
    }
    unsigned short hi[2][4], lo[2][4];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int i = 0; i < 4; ++i) bf16_split(v[r][i], hi[r][i], lo[r][i]);
    // A (row-major 16x16): a0 = (m0, 2t..2t+1), a1 = (m1, 2t..), a2 = (m0, 2t+8..), a3 = (m1, 2t+8..)
    const unsigned ah[4] = {pack2(hi[0][0], hi[0][1]), pack2(hi[1][0], hi[1][1]), pack2(hi[0][2], hi[0][3]),
                            pack2(hi[1][2], hi[1][3])};
    const unsigned al[4] = {pack2(lo[0][0], lo[0][1]), pack2(lo[1][0], lo[1][1]), pack2(lo[0][2], lo[0][3]),
                            pack2(lo[1][2], lo[1][3])};
    // B (col-major 16x8), column grp of tile 0 = row m0 of Jn^T, of tile 1 = row m1
    const unsigned b0h[2] = {pack2(hi[0][0], hi[0][1]), pack2(hi[0][2], hi[0][3])};
    const unsigned b0l[2] = {pack2(lo[0][0], lo[0][1]), pack2(lo[0][2], lo[0][3])};
    const unsigned b1h[2] = {pack2(hi[1][0], hi[1][1]), pack2(hi[1][2], hi[1][3])};
    const unsigned b1l[2] = {pack2(lo[1][0], lo[1][1]), pack2(lo[1][2], lo[1][3])};
    mma_bf16(c0, ah, b0h);
    mma_bf16(c0, ah, b0l);
    mma_bf16(c0, al, b0h);
    mma_bf16(c1, ah, b1h);
    mma_bf16(c1, ah, b1l);
    mma_bf16(c1, al, b1h);
  }
  // C fragment: c[0..1] = (row grp, cols 2t, 2t+1), c[2..3] = (row grp+8, cols 2t, 2t+1)
  double* H = Sl.H + (size_t)s * np * np;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int row = grp + (i >= 2 ? 8 : 0);
    const int colA = 2 * t + (i & 1), colB = 8 + 2 * t + (i & 1);
    // GET_PERTURBATION adds REG_HSS to J^T J (src/lm.f90:173-174)
    const double* rh = Sl.hss ? Sl.hss + (size_t)s * np * np : (C.reg ? C.reg_hss : nullptr);
    if (row < np && colA < np) H[row * np + colA] = (double)c0[i] + (rh ? rh[row * np + colA] : 0.0);
    if (row < np && colB < np) H[row * np + colB] = (double)c1[i] + (rh ? rh[row * np + colB] : 0.0);
  }
  // g = Jn^T r (FP64)
  const double* df = Sl.diff + (size_t)s * nf;
  for (int c = 0; c < np; ++c) {
    const float* rc = J + (size_t)c * nf;
    double acc = 0.0;
    for (int k = lane; k < nf; k += 32) acc += (double)rc[k] * sqrt(w[k]) * df[k];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    // ... and subtracts REG_PEN from J^T r (:169-170)
    if (lane == 0)
      Sl.g[(size_t)s * np + c] = acc * C.norm[c] / sqrt(C.inu) - (Sl.pen ? Sl.pen[(size_t)s * np + c] : 0.0);
  }
}

// One warp per slot, FP64: delta = (H + lambda diag H)^+ g by one-sided
// Jacobi (Hestenes) on the columns of the symmetric matrix, singular values
// below svdtol * max dropped (GET_INVERSE, src/lm.f90:61-133); NaN entries
// of delta are zeroed (NEW_SOLVE_PERTURBATION, src/get_dmodel.f90:806-820).
__global__ void __launch_bounds__(128) k_lm_solve(LMConf C, LMSlots Sl) {
  __shared__ double smA[4][LM_MAXNP][LM_MAXNP + 1], smV[4][LM_MAXNP][LM_MAXNP + 1];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int s = blockIdx.x * (blockDim.x >> 5) + wi;
  if (s >= Sl.S) return;
  if (Sl.pix[s] < 0 || Sl.skip[s]) return;
  const int np = C.np;
  const double lam = Sl.st[5 * (size_t)s + 2];
  const double* H = Sl.H + (size_t)s * np * np;
  double(*A)[LM_MAXNP + 1] = smA[wi];
  double(*V)[LM_MAXNP + 1] = smV[wi];
  // lane i owns row i
  if (lane < np)
    for (int j = 0; j < np; ++j) {
      double h = H[lane * np + j];
      if (j == lane) h = h + h * lam;   // GET_TERM1 (src/lm.f90:43-57)
      A[lane][j] = h;
      V[lane][j] = (lane == j) ? 1.0 : 0.0;
    }
  __syncwarp();
  if (C.solver == 2) {
    // NEW_CALCULATE_DELTA_UBICGSTAB (src/lm.f90:375-453): conjugate gradients
    // on TERM1 delta = TERM2 from delta = 0, stopped when the mean squared
    // relative residual sum(((A x - b)/(|b| + 1e-5))^2)/NP drops below 1e-3
    // (or grows by more than 1e30), at most 100000 iterations; unconverged:
    // x / 10.  A non-finite residual ends the loop at once (its delta would
    // come out non-finite and be zeroed all the same).
    const double b = lane < np ? Sl.g[(size_t)s * np + lane] : 0.0;
    auto dot = [&](double u, double v) {
      double t = lane < np ? u * v : 0.0;
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      return t;
    };
    auto matvec = [&](double v) {
      double t = 0.0;
      for (int j = 0; j < np; ++j) {
        const double vj = __shfl_sync(0xffffffffu, v, j);
        if (lane < np) t += A[lane][j] * vj;
      }
      return t;
    };
    double x = 0.0, pv = b, rv = b;
    double rho = dot(rv, rv);
    double qv = matvec(pv);
    double alpha = rho / dot(pv, qv);
    x += alpha * pv;
    rv -= alpha * qv;
    double pcond = 1.0e29, dcond = -1.0e29;
    bool failed = true;
    for (int it = 1; it <= 100000; ++it) {
      const double rho0 = rho;
      rho = dot(rv, rv);
      const double beta = rho / rho0;
      pv = rv + beta * pv;
      qv = matvec(pv);
      alpha = rho / dot(pv, qv);
      x += alpha * pv;
      rv -= alpha * qv;
      const double ck = matvec(x);
      const double e = (ck - b) / (fabs(b) + 1.0e-5);
      const double cond = dot(e, e) / (double)np;
      if (cond < 1.0e-3 || dcond > 1.0e30) {
        failed = false;
        break;
      }
      if (cond != cond) break;
      dcond = cond - pcond;
      pcond = cond;
    }
    const double d = failed ? x / 10.0 : x;
    if (lane < np) Sl.delta[(size_t)s * np + lane] = (d == d) ? d : 0.0;
    return;
  }
  for (int sweep = 0; sweep < 40; ++sweep) {
    int rot = 0;
    for (int p = 0; p < np - 1; ++p)
      for (int q = p + 1; q < np; ++q) {
        double a = 0.0, b = 0.0, c = 0.0;
        if (lane < np) {
          const double xp = A[lane][p], xq = A[lane][q];
          a = xp * xp;
          b = xq * xq;
          c = xp * xq;
        }
        for (int o = 16; o > 0; o >>= 1) {
          a += __shfl_xor_sync(0xffffffffu, a, o);
          b += __shfl_xor_sync(0xffffffffu, b, o);
          c += __shfl_xor_sync(0xffffffffu, c, o);
        }
        if (fabs(c) > 1e-15 * sqrt(a * b) && c != 0.0) {
          ++rot;
          const double zeta = (b - a) / (2.0 * c);
          const double tt = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          const double cs = 1.0 / sqrt(1.0 + tt * tt), sn = cs * tt;
          if (lane < np) {
            const double xp = A[lane][p], xq = A[lane][q];
            A[lane][p] = cs * xp - sn * xq;
            A[lane][q] = sn * xp + cs * xq;
            const double vp = V[lane][p], vq = V[lane][q];
            V[lane][p] = cs * vp - sn * vq;
            V[lane][q] = sn * vp + cs * vq;
          }
        }
        __syncwarp();
      }
    if (rot == 0) break;
  }
  // sigma_j = |A_j|, u_j = A_j / sigma_j; t_j = u_j.g / sigma_j above the cut
  double sig = 0.0, smax = 0.0;
  double tj = 0.0;
  const double* g = Sl.g + (size_t)s * np;
  for (int j = 0; j < np; ++j) {
    double a = 0.0, u = 0.0;
    if (lane < np) {
      a = A[lane][j] * A[lane][j];
      u = A[lane][j] * g[lane];
    }
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      u += __shfl_xor_sync(0xffffffffu, u, o);
    }
    const double sj = sqrt(a);
    smax = fmax(smax, sj);
    if (lane == j) {
      sig = sj;
      tj = u;   // sigma_j * (u_j . g)
    }
  }
  const double thr = smax * C.svdtol;
  const double coef = (lane < np && sig >= thr && sig > 0.0) ? tj / (sig * sig) : 0.0;
  // delta_i = sum_j V_ij coef_j
  double d = 0.0;
  for (int j = 0; j < np; ++j) {
    const double cj = __shfl_sync(0xffffffffu, coef, j);
    if (lane < np) d += V[lane][j] * cj;
  }
  if (lane < np) Sl.delta[(size_t)s * np + lane] = (d == d) ? d : 0.0;
}

// One CTA per slot: REARANGE_DA_MODEL with SORT_DELTA_TO_ATMOSPHERE
// (NODE_EXPANSION = 1) for every free parameter, then the T taper in log
// tau5 (src/get_dmodel.f90:1975-1989).  coef is the (nz, np) hat table in
// FP64.  MPERT = 0.15 (IFREE_VAR_SPACE, :420).
__global__ void __launch_bounds__(128) k_lm_update(LMConf C, LMSlots Sl, const double* __restrict__ coef) {
  extern __shared__ double sm_upd[];
  const int s = blockIdx.x;
  if (Sl.pix && (Sl.pix[s] < 0 || Sl.skip[s])) return;   // no occupancy arrays: every row is a pixel
  const int nz = C.nz, np = C.np;
  double* nzp = sm_upd;             // nz
  double* avg = nzp + nz;           // np
  double* itd = avg + np;           // np
  double* csum = itd + np;          // np
  float* pert = reinterpret_cast<float*>(csum + np);   // nz
  float* m = Sl.mcur + (size_t)s * 13 * nz;
  const double* delta = Sl.delta + (size_t)s * np;
  const double MPERT = 0.15;
  int j0 = 0;
  for (int rp = 1; rp <= 8; ++rp) {
    const int nj = C.nodes_ref[rp - 1];
    if (nj <= 0) continue;
    const int row = lm_row(C, j0);
    float* ip = m + row * nz;
    const double fac = c_lm_norm[rp - 1], absl = c_lm_norm[rp - 1] * MPERT;
    const double inf = c_lm_low[rp - 1], sup = c_lm_upp[rp - 1];
    // CONTRACT_VECTOR of the current profile, clip of the node deltas
    for (int jj = threadIdx.x; jj < nj; jj += blockDim.x) {
      const int j = j0 + jj;
      double a = 0.0, cs = 0.0;
      for (int k = 0; k < nz; ++k) {
        const double c = coef[k * np + j];
        a += (double)ip[k] * c;
        cs += c;
      }
      a /= cs;
      double pr = fmax(absl, fabs(MPERT * a));
      if (a == 0.0) pr = absl;
      double t = delta[j] * fac;
      if (fabs(t) > pr) t = t / fabs(t) * pr;
      avg[jj] = a;
      itd[jj] = t;
      csum[jj] = cs;
    }
    __syncthreads();
    if (C.node_exp == 2) {
      // NODE_EXPANSION = 2 (STiC-like, :1792-1804): the new profile is the
      // expansion of the clipped node values, limited to [INF, SUP]; the
      // perturbation is its difference to the current profile
      for (int k = threadIdx.x; k < nz; k += blockDim.x) {
        double v = 0.0;
        for (int j = 0; j < nj; ++j) v += (avg[j] + itd[j]) * coef[k * np + j0 + j];
        float op = (float)v;
        if ((double)op < inf) op = (float)inf;
        if ((double)op > sup) op = (float)sup;
        pert[k] = op - ip[k];
      }
      __syncthreads();
    }
    // NZPERT = EXPAND(avg + itd) - IPAR
    for (int k = threadIdx.x; C.node_exp != 2 && k < nz; k += blockDim.x) {
      double v = 0.0;
      for (int j = 0; j < nj; ++j) v += (avg[j] + itd[j]) * coef[k * np + j0 + j];
      nzp[k] = v - (double)ip[k];
    }
    __syncthreads();
    // ITDELTA = CONTRACT(REAL(NZPERT))
    for (int jj = threadIdx.x; C.node_exp != 2 && jj < nj; jj += blockDim.x) {
      const int j = j0 + jj;
      double a = 0.0;
      for (int k = 0; k < nz; ++k) a += (double)(float)nzp[k] * coef[k * np + j];
      itd[jj] = a / csum[jj];
    }
    __syncthreads();
    // NZPERT = EXPAND(ITDELTA), limits
    for (int k = threadIdx.x; C.node_exp != 2 && k < nz; k += blockDim.x) {
      double v = 0.0;
      for (int j = 0; j < nj; ++j) v += itd[j] * coef[k * np + j0 + j];
      const float op = ip[k] + (float)v;
      if (op < inf) v = inf - (double)ip[k];
      if (op > sup) v = sup - (double)ip[k];
      pert[k] = (float)v;
    }
    __syncthreads();
    if (rp == 1 && threadIdx.x == 0) {
      const float* tau = m + 11 * nz;
      const float tll = -11.5f, tul = 0.5f;
      for (int k = nz - 1; k >= 0; --k) {
        if (tau[k] < tll) {
          const float x = fabsf(tau[k] - tll) / 0.5f;
          pert[k] = expf(-(x * x)) * pert[k];
        } else if (tau[k] > tul && k + 1 < nz) {
          pert[k] = pert[k + 1];
        }
      }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nz; k += blockDim.x) ip[k] = pert[k] + ip[k];
    __syncthreads();
    j0 += nj;
  }
}

// One CTA per pixel: the errors mode (GET_ERROR_1D, src/get_dmodel.f90:1248-
// 1287, with NEW_SOLVE_ERRORS :1291-1323).  chi2 of the model's synthesis
// (NEW_CALCULATE_CHI2 :960-983, penalties included under regularisation),
// the diagonal of H = Jn^T Jn of the normalised Jacobian (NORMALIZE_JACOB,
// FP64 over the REAL*4 EQVDSYN), per node sigma_i = sqrt((chi2/INU)/H_ii)
// (1e32 where H_ii <= 1e-32), then REARANGE_DA_MODEL in its errors form on a
// zeroed model (:1877-1883: limits 0 and 1e20; the clip of SORT_DELTA at
// PARAM_NORM * MPERT since the zero model's node averages are 0; the T taper
// reads log tau5 = 0 and so leaves the profile alone).  err: MODEL(NZ,13),
// rows of fixed parameters zero, as ESPLIT_MODEL3D receives it (:291-334).
// Dynamic shared memory: nz doubles + nz floats.
__global__ void __launch_bounds__(256) k_lm_errors(LMConf C, int n, const double* __restrict__ obs,
                                                   const double* __restrict__ syn, const float* __restrict__ jac,
                                                   const float* __restrict__ model, const double* __restrict__ w,
                                                   const double* __restrict__ coef, float* __restrict__ err,
                                                   double* __restrict__ chi_out) {
  extern __shared__ double sm_err[];
  __shared__ double red[8];
  __shared__ double xs[LM_MAXNP], pr[LM_MAXNP], hd[LM_MAXNP], itd[LM_MAXNP], csum[LM_MAXNP];
  __shared__ double nume;
  const int p = blockIdx.x;
  if (p >= n) return;
  const int nf = C.nfreq, np = C.np, nz = C.nz, nm = 13 * nz;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const double* o = obs + (size_t)p * nf;
  const double* sy = syn + (size_t)p * nf;
  double e = 0.0;
  for (int i = threadIdx.x; i < nf; i += blockDim.x) {
    const double d = o[i] - sy[i];
    e += d * d * w[i];
  }
  double chi = block_sum_d(e, red) / C.inu;
  if (C.reg) {
    const float* m = model + (size_t)p * nm;
    if (threadIdx.x < np) xs[threadIdx.x] = lm_node_value(C, m, coef, threadIdx.x);
    __syncthreads();
    if (threadIdx.x < np) pr[threadIdx.x] = lm_pen_res(C, xs, threadIdx.x);
    __syncthreads();
    double pp = 0.0;
    for (int j = 0; j < np; ++j) pp += pr[j] * pr[j];
    chi += pp;
  }
  // H_ii: one warp per node, FP64 sums over the frequencies
  const float* J = jac + (size_t)p * np * nf;
  const double rin = 1.0 / sqrt(C.inu);
  for (int j = warp; j < np; j += nwarp) {
    double h = 0.0;
    for (int f = lane; f < nf; f += 32) {
      const double t = (double)J[(size_t)j * nf + f] * (sqrt(w[f]) * rin) * C.norm[j];
      h += t * t;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) h += __shfl_xor_sync(0xffffffffu, h, off);
    if (lane == 0) hd[j] = h;
  }
  if (threadIdx.x == 0) {
    chi_out[p] = chi;
    nume = chi / C.inu;
  }
  __syncthreads();
  double* nzp = sm_err;                                  // nz
  float* pert = reinterpret_cast<float*>(nzp + nz);      // nz
  float* out = err + (size_t)p * nm;
  for (int i = threadIdx.x; i < nm; i += blockDim.x) out[i] = 0.0f;
  __syncthreads();
  const double MPERT = 0.15;
  int j0 = 0;
  for (int rp = 1; rp <= 8; ++rp) {
    const int nj = C.nodes_ref[rp - 1];
    if (nj <= 0) continue;
    const int row = C.row_of[j0];
    const double absl = c_lm_norm[rp - 1] * MPERT;
    if (threadIdx.x < nj) {
      const int j = j0 + threadIdx.x;
      const double sig = hd[j] > 1.0e-32 ? sqrt(nume / hd[j]) : 1.0e32;
      double cs = 0.0;
      for (int k = 0; k < nz; ++k) cs += coef[k * np + j];
      double t = sig * c_lm_norm[rp - 1];
      if (fabs(t) > absl) t = t / fabs(t) * absl;
      itd[threadIdx.x] = t;
      csum[threadIdx.x] = cs;
    }
    __syncthreads();
    // NZPERT = EXPAND(0 + ITDELTA) - 0
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
      double v = 0.0;
      for (int j = 0; j < nj; ++j) v += itd[j] * coef[k * np + j0 + j];
      nzp[k] = v;
    }
    __syncthreads();
    // ITDELTA = CONTRACT(REAL(NZPERT))
    if (threadIdx.x < nj) {
      const int j = j0 + threadIdx.x;
      double a = 0.0;
      for (int k = 0; k < nz; ++k) a += (double)(float)nzp[k] * coef[k * np + j];
      itd[threadIdx.x] = a / csum[threadIdx.x];
    }
    __syncthreads();
    // NZPERT = EXPAND(ITDELTA), limits [0, 1e20] on 0 + NZPERT
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
      double v = 0.0;
      for (int j = 0; j < nj; ++j) v += itd[j] * coef[k * np + j0 + j];
      const float op = (float)v;
      if (op < 0.0f) v = 0.0;
      if (op > 1.0e20f) v = 1.0e20;
      pert[k] = (float)v;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nz; k += blockDim.x) out[row * nz + k] = pert[k];
    __syncthreads();
    j0 += nj;
  }
}

// One CTA per slot: the field-wide stop of MAKE_DECISION (src/invert3d.f90:
// 843-846) ends every pixel still in flight; each writes its best model out
// as a finished pixel does (END_CYCLE).
__global__ void __launch_bounds__(256) k_lm_finish_all(LMConf C, LMSlots Sl, LMQueue* q, float* __restrict__ out_model,
                                                       double* __restrict__ out_chi, int* __restrict__ out_iter,
                                                       double* __restrict__ out_syn, int* __restrict__ out_status) {
  const int s = blockIdx.x;
  const int p = Sl.pix[s];
  if (p < 0) return;
  const int nf = C.nfreq, nm = 13 * C.nz;
  const double* st = Sl.st + 5 * (size_t)s;
  const float* mb = Sl.mbest + (size_t)s * nm;
  for (int i = threadIdx.x; i < nm; i += blockDim.x) out_model[(size_t)p * nm + i] = mb[i];
  if (out_syn)
    for (int i = threadIdx.x; i < nf; i += blockDim.x) out_syn[(size_t)p * nf + i] = Sl.synb[(size_t)s * nf + i];
  if (threadIdx.x == 0) {
    out_chi[p] = st[1];
    out_iter[p] = Sl.iter[s] + (Sl.restarted[s] > 0 ? Sl.restarted[s] - 1 : 0);
    if (out_status) out_status[p] = st[1] < 1.0e29 ? 0 : FZ_NAN;
    lm_state_out(C, st, p);
    atomicAdd(&q->done, 1);
    Sl.pix[s] = LM_PAD;
  }
}

// One block of 1024 threads: destination of every occupied slot when the
// pool is compacted (exclusive scan of the occupancy flags), and their count.
__global__ void __launch_bounds__(1024) k_lm_scan(int S, const int* __restrict__ pix, int* __restrict__ dest,
                                                  LMQueue* q, int* __restrict__ list = nullptr) {
  __shared__ int part[1024];
  const int per = (S + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per, e = min(S, b + per);
  int n = 0;
  for (int i = b; i < e; ++i) n += pix[i] >= 0;
  part[threadIdx.x] = n;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {   // inclusive Hillis-Steele scan
    const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int d = part[threadIdx.x] - n;
  for (int i = b; i < e; ++i) {
    const bool occ = pix[i] >= 0;
    if (occ && list) list[d] = i;   // the occupied slots in order
    dest[i] = occ ? d++ : -1;
  }
  if (threadIdx.x == blockDim.x - 1) q->active = part[threadIdx.x];
}

// The condition of the device-driven inversion loop (a CUDA graph WHILE
// node around one iteration): another iteration while pixels are left, no
// tensor-core kernel gave up and fewer than cap iterations ran; with gthr >
// 0, MAKE_DECISION's field-wide stop (mean STEPS >= gthr,
// src/invert3d.f90:843-846) ends the loop with gstop set, and the host then
// finishes every pixel in flight.
__global__ void k_lm_ctl(LMQueue* q, cudaGraphConditionalHandle h, int npix, long long cap, int gthr) {
  const int it = ++q->iters;
  unsigned go;
  if (q->done >= npix || q->tc_err) {
    go = 0u;
  } else if (gthr > 0 && (double)(long long)q->steps_sum >= (double)gthr * (double)npix) {
    q->gstop = 1;
    go = 0u;
  } else {
    go = it < cap ? 1u : 0u;
  }
  cudaGraphSetConditional(h, go);
}

// One block of 1024 threads: the slots of the RF pass (need_rf) compacted
// into rf_list, and their count.
__global__ void __launch_bounds__(1024) k_lm_rflist(int S, const int* __restrict__ need, int* __restrict__ list,
                                                    LMQueue* q) {
  __shared__ int part[1024];
  const int per = (S + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per, e = min(S, b + per);
  int n = 0;
  for (int i = b; i < e; ++i) n += need[i] != 0;
  part[threadIdx.x] = n;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {   // inclusive Hillis-Steele scan
    const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int d = part[threadIdx.x] - n;
  for (int i = b; i < e; ++i)
    if (need[i]) list[d++] = i;
  if (threadIdx.x == blockDim.x - 1) q->rf_count = part[threadIdx.x];
}

// One CTA per source slot: copy an occupied slot to its compacted position
// in the other pool (the state the next iteration reads).
__global__ void __launch_bounds__(256) k_lm_compact(LMConf C, LMSlots A, LMSlots B, const int* __restrict__ dest) {
  const int s = blockIdx.x, d = dest[s];
  if (d < 0) return;
  const int nf = C.nfreq, nm = 13 * C.nz;
  if (threadIdx.x == 0) {
    B.pix[d] = A.pix[s];
    B.iter[d] = A.iter[s];
    B.skip[d] = A.skip[s];
    B.restarted[d] = A.restarted[s];
  }
  if (threadIdx.x < 5) B.st[5 * (size_t)d + threadIdx.x] = A.st[5 * (size_t)s + threadIdx.x];
  for (int i = threadIdx.x; i < nm; i += blockDim.x) {
    B.mcur[(size_t)d * nm + i] = A.mcur[(size_t)s * nm + i];
    B.mbest[(size_t)d * nm + i] = A.mbest[(size_t)s * nm + i];
  }
  for (int i = threadIdx.x; i < nf; i += blockDim.x) {
    B.synb[(size_t)d * nf + i] = A.synb[(size_t)s * nf + i];
    B.obs[(size_t)d * nf + i] = A.obs[(size_t)s * nf + i];
  }
  const float4* ja = reinterpret_cast<const float4*>(A.jacb + (size_t)s * C.np * nf);
  float4* jb = reinterpret_cast<float4*>(B.jacb + (size_t)d * C.np * nf);
  for (int i = threadIdx.x; i < C.np * nf / 4; i += blockDim.x) jb[i] = ja[i];
  if (C.np <= LM_MAXNP) {
    // the warp normal equations run on accepted steps only: H and g travel
    // with the slot (the tensor-core ones are rebuilt every iteration)
    const int np = C.np;
    for (int i = threadIdx.x; i < np * np; i += blockDim.x) B.H[(size_t)d * np * np + i] = A.H[(size_t)s * np * np + i];
    for (int i = threadIdx.x; i < np; i += blockDim.x) B.g[(size_t)d * np + i] = A.g[(size_t)s * np + i];
  }
}

}  // namespace
