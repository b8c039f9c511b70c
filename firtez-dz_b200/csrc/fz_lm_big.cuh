// Batched LM for node layouts larger than the warp kernels' 16 nodes
// (sm_100a), included by fz_cuda.cu after fz_lm.cuh.  The reference's
// default schedule frees every height of a parameter in its last cycle
// (GET_NJEVALS / UPDATE_COEFS, src/get_dmodel.f90:377-721), NP in the
// hundreds; its only inversion test runs T and v_z at all 256 heights
// (NP = 512).  Per slot:
//   k_rf_contract  the node Jacobian from the response functions at every
//                  height: J(node j of p) = sum_k coef(k, j) RF_p(k), the
//                  contraction of CALCULATE_EQUIVALENT_DSYN
//                  (src/forward.f90:552-681) on the full RFs;
//   k_lm_gram_tc   H = Jn Jn^T on the fifth-generation tensor cores: the
//                  normalised FP32 Jacobian split into bf16 hi + lo parts
//                  while it is staged in shared memory, hi hi^T + hi lo^T +
//                  lo hi^T accumulated in FP32 in tensor memory
//                  (tcgen05.mma, M = 128 tiles, upper-triangle tile pairs);
//   k_lm_grad      g = Jn^T r in FP64 (HESSIAN / GET_TERM1's TERM2,
//                  src/lm.f90:30-57, with REG_PEN / REG_HSS);
//   k_lm_cg_big    NEW_CALCULATE_DELTA_UBICGSTAB (src/lm.f90:375-453), one
//                  CTA per slot, FP64, H in global memory;
//   k_lm_svd_big   GET_INVERSE's pseudo-inverse (src/lm.f90:61-133) by a
//                  one-sided Jacobi SVD in FP64 (round-robin pair order, one
//                  CTA per slot, the columns in global memory).
#pragma once

#include "fz_tc.cuh"

namespace {

constexpr int GT_M = 128;                       // tile rows = TMEM lanes
constexpr int GT_BK = 64;                       // bf16 K elements per stage
constexpr int GT_NKC = GT_BK / 8;               // core-matrix columns per 8-row group
constexpr int GT_TILE = GT_M * GT_BK * 2;       // bytes of one bf16 tile (16 KB)
constexpr int GT_STAGE = 4 * GT_TILE;           // A hi, A lo, B hi, B lo
constexpr size_t GT_SMEM = 2 * (size_t)GT_STAGE;   // two stages (128 KB)
constexpr unsigned long long GT_WAIT_NS = 2000000000ull;   // 2 s per wait on the tensor core

// Stage rows [row0, row0 + 128) x K block [k0, k0 + 64) of the slot's
// Jacobian J (np, nf) into the hi / lo bf16 tiles, normalised as
// NORMALIZE_JACOB does (wk = sqrt(w / INU) of the block's frequencies, from
// shared memory, and PARAM_NORM per node); rows >= np and frequencies >= nf
// are zero.
__device__ __forceinline__ void gram_stage(const LMConf& C, const float* __restrict__ J, const float* wk, int row0,
                                           int k0, unsigned char* hi, unsigned char* lo) {
  // blocks of 128 threads: 16 float4 of the tile a thread, all loads issued
  // before any is used
  constexpr int PER = GT_M * (GT_BK / 4) / 128;
  const int np = C.np, nf = C.nfreq;
  float4 x[PER];
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int i = threadIdx.x + 128 * u;
    const int gr = row0 + (i >> 4), k = k0 + 4 * (i & 15);
    x[u] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (gr < np) {
      const float* src = J + (size_t)gr * nf + k;
      if (k + 4 <= nf) {
        x[u] = __ldg(reinterpret_cast<const float4*>(src));
      } else {
        float t[4] = {0.f, 0.f, 0.f, 0.f};
        for (int e = 0; e < 4; ++e)
          if (k + e < nf) t[e] = src[e];
        x[u] = make_float4(t[0], t[1], t[2], t[3]);
      }
    }
  }
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int i = threadIdx.x + 128 * u;
    const int r = i >> 4, kq = i & 15;
    const int gr = row0 + r;
    const float nrm = gr < np ? (float)lm_nrm(C, gr) : 0.f;
    const float v[4] = {x[u].x * wk[4 * kq] * nrm, x[u].y * wk[4 * kq + 1] * nrm, x[u].z * wk[4 * kq + 2] * nrm,
                        x[u].w * wk[4 * kq + 3] * nrm};
    unsigned short h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) bf16_split(v[e], h[e], l[e]);
    const uint32_t off = fztc::kmajor_offset(r, 4 * kq, GT_NKC);
    *reinterpret_cast<uint2*>(hi + off) = make_uint2(pack2(h[0], h[1]), pack2(h[2], h[3]));
    *reinterpret_cast<uint2*>(lo + off) = make_uint2(pack2(l[0], l[1]), pack2(l[2], l[3]));
  }
}

// One CTA of 128 threads per (tile pair bi <= bj, slot): the 128 x 128 block
// (bi, bj) of H = Jn Jn^T (+ PEN_HSS), written to both triangles in FP64.
// A wait that runs out sets *err and ends the CTA after freeing its tensor
// memory.
__global__ void __launch_bounds__(128, 1) k_lm_gram_tc(LMConf C, LMSlots Sl, const double* __restrict__ w,
                                                       int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char gsm[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tbase;
  __shared__ float wk[2][GT_BK];   // sqrt(w / INU) of the K block's frequencies, per buffer
  const int s = blockIdx.y;
  if (Sl.pix[s] < 0 || Sl.skip[s]) return;
  const int np = C.np, nf = C.nfreq;
  const int nb = (np + GT_M - 1) / GT_M;
  int t = blockIdx.x, bi = 0;
  while (bi < nb && t >= nb - bi) {
    t -= nb - bi;
    ++bi;
  }
  if (bi >= nb) return;
  const int bj = bi + t;
  const bool diag = bi == bj;
  const int r0 = bi * GT_M, c0 = bj * GT_M;
  const int nrB = min(GT_M, np - c0);
  const int N = (nrB + 15) & ~15;   // 16 .. 128
  const float* J = Sl.jacb + (size_t)s * np * nf;
  const float rin = (float)(1.0 / sqrt(C.inu));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    fztc::tmem_alloc(&tbase, 128);
    fztc::tmem_relinquish();
  }
  if (tid == 0) {
    fztc::mbar_init(&mbar[0], 1);
    fztc::mbar_init(&mbar[1], 1);
    fztc::fence_mbar_init();
  }
  fztc::fence_before_sync();
  __syncthreads();
  fztc::fence_after_sync();
  const uint32_t tmem = tbase;
  const uint32_t idesc = fztc::idesc_bf16(GT_M, N);
  const int nkb = (nf + GT_BK - 1) / GT_BK;
  bool ok = true;
  for (int kb = 0; kb < nkb && ok; ++kb) {
    const int buf = kb & 1;
    unsigned char* ah = gsm + (size_t)buf * GT_STAGE;
    unsigned char* al = ah + GT_TILE;
    unsigned char* bh = diag ? ah : ah + 2 * GT_TILE;
    unsigned char* bl = diag ? al : ah + 3 * GT_TILE;
    // the tensor core has finished reading this buffer (block kb - 2)
    if (kb >= 2) ok = fztc::mbar_wait(&mbar[buf], ((kb - 2) >> 1) & 1, GT_WAIT_NS);
    if (tid < GT_BK) {
      const int k = kb * GT_BK + tid;
      wk[buf][tid] = k < nf ? sqrtf((float)w[k]) * rin : 0.f;
    }
    ok = __syncthreads_and(ok);
    if (!ok) break;
    gram_stage(C, J, wk[buf], r0, kb * GT_BK, ah, al);
    if (!diag) gram_stage(C, J, wk[buf], c0, kb * GT_BK, bh, bl);
    fztc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      const uint32_t sah = fztc::smem_addr(ah), sal = fztc::smem_addr(al);
      const uint32_t sbh = fztc::smem_addr(bh), sbl = fztc::smem_addr(bl);
#pragma unroll
      for (int ks = 0; ks < GT_BK / 16; ++ks) {
        const uint32_t o = ks * 256;   // two core-matrix columns of K
        const uint64_t dah = fztc::desc_kmajor(sah + o, 128, GT_NKC * 128);
        const uint64_t dal = fztc::desc_kmajor(sal + o, 128, GT_NKC * 128);
        const uint64_t dbh = fztc::desc_kmajor(sbh + o, 128, GT_NKC * 128);
        const uint64_t dbl = fztc::desc_kmajor(sbl + o, 128, GT_NKC * 128);
        fztc::mma_bf16(tmem, dah, dbh, idesc, (kb > 0 || ks > 0) ? 1u : 0u);
        fztc::mma_bf16(tmem, dah, dbl, idesc, 1u);
        fztc::mma_bf16(tmem, dal, dbh, idesc, 1u);
      }
      fztc::commit(&mbar[buf]);
    }
  }
  if (ok) {
    const int last = nkb - 1;
    ok = fztc::mbar_wait(&mbar[last & 1], (last >> 1) & 1, GT_WAIT_NS);
  }
  ok = __syncthreads_and(ok);
  fztc::fence_after_sync();
  if (ok) {
    const int r = warp * 32 + lane;   // tile row = TMEM lane
    const int gr = r0 + r;
    const double* rh = Sl.hss ? Sl.hss + (size_t)s * np * np : nullptr;
    double* H = Sl.H + (size_t)s * np * np;
    for (int cc = 0; cc < N; cc += 16) {
      float v[16];
      fztc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cc, v);
      if (gr >= np) continue;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int gc = c0 + cc + i;
        if (gc >= np || (diag && gc < gr)) continue;
        // GET_PERTURBATION adds REG_HSS to J^T J (src/lm.f90:173-174)
        const double h = (double)v[i] + (rh ? rh[(size_t)gr * np + gc] : (C.reg ? lm_hss(C, gr, gc) : 0.0));
        const double ht = (double)v[i] + (rh ? rh[(size_t)gc * np + gr] : (C.reg ? lm_hss(C, gc, gr) : 0.0));
        H[(size_t)gr * np + gc] = h;
        H[(size_t)gc * np + gr] = ht;
      }
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  fztc::fence_before_sync();
  __syncthreads();
  if (warp == 0) fztc::tmem_dealloc(tmem, 128);
}

// g_c = Jn_c . r in FP64 minus REG_PEN (src/lm.f90:165-170); one warp per
// (slot, node).
__global__ void __launch_bounds__(256) k_lm_grad(LMConf C, LMSlots Sl, const double* __restrict__ w) {
  const int s = blockIdx.y;
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= C.np || Sl.pix[s] < 0 || Sl.skip[s]) return;
  const int nf = C.nfreq, np = C.np;
  const float* rc = Sl.jacb + ((size_t)s * np + c) * nf;
  const double* df = Sl.diff + (size_t)s * nf;
  double acc = 0.0;
  for (int k = lane; k < nf; k += 32) acc += (double)rc[k] * sqrt(w[k]) * df[k];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0)
    Sl.g[(size_t)s * np + c] = acc * lm_nrm(C, c) / sqrt(C.inu) - (Sl.pen ? Sl.pen[(size_t)s * np + c] : 0.0);
}

__device__ __forceinline__ double cta_sum_d(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < nw; ++i) t += red[i];
  return t;
}

// y = TERM1 v with TERM1 = H + lambda diag H (GET_TERM1, src/lm.f90:43-57):
// one warp per row, lanes over the columns.
__device__ __forceinline__ void big_matvec(const double* __restrict__ H, int np, double lam, const double* v,
                                           double* y) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int i = warp; i < np; i += nw) {
    const double* hr = H + (size_t)i * np;
    double t = 0.0;
    for (int j = lane; j < np; j += 32) t += hr[j] * v[j];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) y[i] = t + hr[i] * lam * v[i];
  }
  __syncthreads();
}

// NEW_CALCULATE_DELTA_UBICGSTAB on TERM1 delta = TERM2 from delta = 0, as the
// warp kernel: stop when the mean squared relative residual drops below
// 1e-3 (or grows by more than 1e30), at most 100000 iterations, x / 10 when
// unconverged, a non-finite residual ends the loop; NaN entries zeroed.
// One CTA per slot, dynamic shared memory 6 np doubles.
__global__ void __launch_bounds__(256) k_lm_cg_big(LMConf C, LMSlots Sl) {
  extern __shared__ double cgs[];
  __shared__ double red[8];
  const int s = blockIdx.x;
  if (Sl.pix[s] < 0 || Sl.skip[s]) return;
  const int np = C.np;
  const double lam = Sl.st[5 * (size_t)s + 2];
  const double* H = Sl.H + (size_t)s * np * np;
  double *b = cgs, *x = b + np, *pv = x + np, *rv = pv + np, *qv = rv + np, *ck = qv + np;
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    const double g = Sl.g[(size_t)s * np + i];
    b[i] = g;
    x[i] = 0.0;
    pv[i] = g;
    rv[i] = g;
  }
  __syncthreads();
  auto dot = [&](const double* u, const double* v) {
    double t = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) t += u[i] * v[i];
    return cta_sum_d(t, red);
  };
  double rho = dot(rv, rv);
  big_matvec(H, np, lam, pv, qv);
  double alpha = rho / dot(pv, qv);
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    x[i] += alpha * pv[i];
    rv[i] -= alpha * qv[i];
  }
  __syncthreads();
  double pcond = 1.0e29, dcond = -1.0e29;
  bool failed = true;
  for (int it = 1; it <= 100000; ++it) {
    const double rho0 = rho;
    rho = dot(rv, rv);
    const double beta = rho / rho0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) pv[i] = rv[i] + beta * pv[i];
    __syncthreads();
    big_matvec(H, np, lam, pv, qv);
    alpha = rho / dot(pv, qv);
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
      x[i] += alpha * pv[i];
      rv[i] -= alpha * qv[i];
    }
    __syncthreads();
    big_matvec(H, np, lam, x, ck);
    double e2 = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
      const double e = (ck[i] - b[i]) / (fabs(b[i]) + 1.0e-5);
      e2 += e * e;
    }
    const double cond = cta_sum_d(e2, red) / (double)np;
    if (cond < 1.0e-3 || dcond > 1.0e30) {
      failed = false;
      break;
    }
    if (cond != cond) break;
    dcond = cond - pcond;
    pcond = cond;
  }
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    const double d = failed ? x[i] / 10.0 : x[i];
    Sl.delta[(size_t)s * np + i] = (d == d) ? d : 0.0;
  }
}

// Member m (0..n-1) of round r of the round-robin pairing of n players
// (n even): player 0 stays, the others rotate.
__device__ __forceinline__ int rr_member(int m, int r, int n) { return m == 0 ? 0 : ((m - 1 + r) % (n - 1)) + 1; }

// GET_INVERSE's pseudo-inverse applied to TERM2 (src/lm.f90:61-204): a
// one-sided Jacobi SVD of TERM1 = H + lambda diag H (symmetric; its columns
// are its rows) in FP64, the rotations of a round applied to disjoint column
// pairs in parallel, sweeps until none rotates (at most 40); singular values
// below svdtol x the largest dropped; NaN entries of delta zeroed.  One CTA
// per slot; A and V (np x np, column-major) in the slot's scratch.
__global__ void __launch_bounds__(256) k_lm_svd_big(LMConf C, LMSlots Sl, double* __restrict__ scratch) {
  __shared__ int rot;
  __shared__ double red[8];
  extern __shared__ double svs[];   // coef (np)
  const int s = blockIdx.x;
  if (Sl.pix[s] < 0 || Sl.skip[s]) return;
  const int np = C.np, npad = np + (np & 1);
  const double lam = Sl.st[5 * (size_t)s + 2];
  const double* H = Sl.H + (size_t)s * np * np;
  double* A = scratch + (size_t)s * 2 * np * np;
  double* V = A + (size_t)np * np;
  for (size_t i = threadIdx.x; i < (size_t)np * np; i += blockDim.x) {
    const int r = (int)(i / np), c = (int)(i % np);
    double h = H[i];
    if (r == c) h = h + h * lam;   // GET_TERM1
    A[i] = h;                      // column r, row c (symmetric)
    V[i] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int sweep = 0; sweep < 40; ++sweep) {
    if (threadIdx.x == 0) rot = 0;
    __syncthreads();
    for (int r = 0; r < npad - 1; ++r) {
      for (int k = warp; k < npad / 2; k += nw) {
        int p = rr_member(k, r, npad), q = rr_member(npad - 1 - k, r, npad);
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        if (q >= np) continue;   // the padding column of an odd count
        double* ap = A + (size_t)p * np;
        double* aq = A + (size_t)q * np;
        double a = 0.0, b = 0.0, c = 0.0;
        for (int i = lane; i < np; i += 32) {
          const double xp = ap[i], xq = aq[i];
          a += xp * xp;
          b += xq * xq;
          c += xp * xq;
        }
        for (int o = 16; o > 0; o >>= 1) {
          a += __shfl_xor_sync(0xffffffffu, a, o);
          b += __shfl_xor_sync(0xffffffffu, b, o);
          c += __shfl_xor_sync(0xffffffffu, c, o);
        }
        if (fabs(c) > 1e-15 * sqrt(a * b) && c != 0.0) {
          if (lane == 0) rot = 1;
          const double zeta = (b - a) / (2.0 * c);
          const double tt = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          const double cs = 1.0 / sqrt(1.0 + tt * tt), sn = cs * tt;
          double* vp = V + (size_t)p * np;
          double* vq = V + (size_t)q * np;
          for (int i = lane; i < np; i += 32) {
            const double xp = ap[i], xq = aq[i];
            ap[i] = cs * xp - sn * xq;
            aq[i] = sn * xp + cs * xq;
            const double yp = vp[i], yq = vq[i];
            vp[i] = cs * yp - sn * yq;
            vq[i] = sn * yp + cs * yq;
          }
        }
      }
      __syncthreads();
    }
    const bool any = rot != 0;
    __syncthreads();   // every thread has read the flag before it is reset
    if (!any) break;
  }
  // sigma_j = |A_j|, coef_j = (A_j . g) / sigma_j^2 above the cut
  const double* g = Sl.g + (size_t)s * np;
  double smax = 0.0;
  for (int j = warp; j < np; j += nw) {
    const double* aj = A + (size_t)j * np;
    double a = 0.0, u = 0.0;
    for (int i = lane; i < np; i += 32) {
      a += aj[i] * aj[i];
      u += aj[i] * g[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      u += __shfl_xor_sync(0xffffffffu, u, o);
    }
    if (lane == 0) {
      svs[j] = sqrt(a);                    // sigma_j for now
      svs[np + j] = u;                     // sigma_j (u_j . g)
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < np; j += blockDim.x) smax = fmax(smax, svs[j]);
  for (int o = 16; o > 0; o >>= 1) smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
  __syncthreads();
  if (lane == 0) red[warp] = smax;
  __syncthreads();
  smax = 0.0;
  for (int i = 0; i < nw; ++i) smax = fmax(smax, red[i]);
  const double thr = smax * C.svdtol;
  __syncthreads();
  for (int j = threadIdx.x; j < np; j += blockDim.x) {
    const double sj = svs[j];
    svs[j] = (sj >= thr && sj > 0.0) ? svs[np + j] / (sj * sj) : 0.0;
  }
  __syncthreads();
  // delta_i = sum_j V_ij coef_j (V column j holds V(:, j))
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    double d = 0.0;
    for (int j = 0; j < np; ++j) d += V[(size_t)j * np + i] * svs[j];
    Sl.delta[(size_t)s * np + i] = (d == d) ? d : 0.0;
  }
}

// The node Jacobian from the response functions at every height of the
// listed columns: jac(col, n0[p] + j, f) = sum_k coef(k, n0[p] + j)
// rf(col, p, k, f) (rf already x GAIN); one thread per frequency.
__global__ void __launch_bounds__(256) k_rf_contract(int nz, int nf, RFConf R, const float* __restrict__ coef,
                                                     const float* __restrict__ rf, float* __restrict__ jac,
                                                     const int* __restrict__ list, const int* __restrict__ nlist) {
  const int np = R.np;
  if (list && (int)blockIdx.z >= *nlist) return;
  const int col = list ? list[blockIdx.z] : (int)blockIdx.z;
  const int node = blockIdx.y;
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  int p = 0;
  while (p < NSLOT - 1 && node >= R.n0[p] + R.nj[p]) ++p;
  const float* src = rf + ((size_t)col * 6 + p) * nz * nf + f;
  float acc = 0.0f;
  for (int k = 0; k < nz; ++k) {
    const float c = coef[(size_t)k * np + node];
    if (c != 0.0f) acc = fmaf(c, src[(size_t)k * nf], acc);
  }
  jac[((size_t)col * np + node) * nf + f] = acc;
}

}  // namespace
