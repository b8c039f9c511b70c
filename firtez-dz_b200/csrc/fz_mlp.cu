// Warm-start network of the inversion: an MLP from the observed Stokes vector
// to the node values of the model, trained and run with hand-written BF16
// kernels (sm_100a): tcgen05 tensor-core GEMMs (bf16 operands, FP32
// accumulation in tensor memory) with fused bias / GELU / GELU' epilogues,
// an MSE loss kernel and Adam on FP32 master weights.  It has no counterpart in the reference,
// whose initial guess is the model in the control file (or the Stokes-moment
// assists of SET_TAU, src/invert3d.f90:492-727).
//
// Layouts: activations row-major [batch][features] in bf16; weights W[out][in]
// row-major (bf16 copy for the GEMMs, FP32 master for Adam); biases FP32.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/fz_b200.h"
#include "fz_tc.cuh"

namespace {

constexpr int MLP_MAXL = 8;

enum GemmMode { NT = 0, NN = 1, TN = 2 };
enum Epi { EPI_FWD_GELU = 0, EPI_FWD_LIN = 1, EPI_BWD_GELU = 2, EPI_F32 = 3 };

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
  return cdf + z * pdf;
}

// C (M x N) = A B^T with the logical operands of each mode:
//   NT: A[m][k] = a[m*lda + k],  B[n][k] = b[n*ldb + k]   (Y = X W^T)
//   NN: A[m][k] = a[m*lda + k],  B[n][k] = b[k*ldb + n]   (dX = dZ W)
//   TN: A[m][k] = a[k*lda + m],  B[n][k] = b[k*ldb + n]   (dW = dZ^T X)
// and the epilogues
//   EPI_FWD_GELU: z = C + bias[n] -> zout (fp32, pre-activation), out = bf16(gelu(z))
//   EPI_FWD_LIN : z = C + bias[n] -> fout (fp32)
//   EPI_BWD_GELU: out = bf16(C * gelu'(zin[m][n]))
//   EPI_F32     : fout = C (fp32)
// on the fifth-generation tensor cores (tcgen05): a 128 x 128
// output tile per CTA of 256 threads, K in blocks of 64 staged into shared
// memory in the canonical K-major layout (fz_tc.cuh) through three buffers,
// one elected thread issuing tcgen05.mma (bf16 x bf16 -> FP32 in tensor
// memory) and committing each block to the buffer's mbarrier, the epilogue
// read back with tcgen05.ld (warps w and w + 4 share TMEM lanes 32 (w % 4)..,
// columns 0-63 and 64-127).  Operands whose leading dimension allows it move
// in 16-byte vectors, the others element by element.
constexpr int TC_BK = 64, TC_NKC = TC_BK / 8, TC_STAGES = 3;
constexpr int TC_TILE = 128 * TC_BK * 2;                      // one 128 x 64 bf16 tile
constexpr size_t TC_SMEM = (size_t)TC_STAGES * 2 * TC_TILE;   // A and B per stage: 96 KB
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;

// Rows [row0, row0 + 128) x K [k0, k0 + 64) of a logical operand X (R x K)
// stored K-contiguous (X[r * ld + k], kcont) or row-contiguous (X[k * ld +
// r]) into the K-major tile dst; out-of-range elements are zero.
__device__ __forceinline__ void tc_stage(const __nv_bfloat16* __restrict__ X, int ld, bool kcont, bool vec, int row0,
                                         int k0, int R, int K, unsigned char* dst) {
  const unsigned short* x = reinterpret_cast<const unsigned short*>(X);
  if (kcont) {
    for (int i = threadIdx.x; i < 128 * (TC_BK / 8); i += blockDim.x) {
      const int r = i / (TC_BK / 8), c = i % (TC_BK / 8);
      const int gr = row0 + r, gk = k0 + 8 * c;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (gr < R) {
        const unsigned short* src = x + (size_t)gr * ld + gk;
        if (vec && gk + 8 <= K) {
          v = *reinterpret_cast<const uint4*>(src);
        } else {
          unsigned short e[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) e[j] = gk + j < K ? src[j] : (unsigned short)0;
          v = make_uint4(e[0] | ((unsigned)e[1] << 16), e[2] | ((unsigned)e[3] << 16), e[4] | ((unsigned)e[5] << 16),
                         e[6] | ((unsigned)e[7] << 16));
        }
      }
      *reinterpret_cast<uint4*>(dst + fztc::kmajor_offset(r, 8 * c, TC_NKC)) = v;
    }
  } else {
    for (int i = threadIdx.x; i < TC_BK * 16; i += blockDim.x) {
      const int kk = i / 16, c = i % 16;   // eight consecutive rows 8c.. at one k
      const int gk = k0 + kk, gr = row0 + 8 * c;
      unsigned short e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (gk < K) {
        const unsigned short* src = x + (size_t)gk * ld + gr;
        if (vec && gr + 8 <= R) {
          const uint4 v = *reinterpret_cast<const uint4*>(src);
          e[0] = v.x & 0xffff; e[1] = v.x >> 16; e[2] = v.y & 0xffff; e[3] = v.y >> 16;
          e[4] = v.z & 0xffff; e[5] = v.z >> 16; e[6] = v.w & 0xffff; e[7] = v.w >> 16;
        } else {
#pragma unroll
          for (int j = 0; j < 8; ++j) e[j] = gr + j < R ? src[j] : (unsigned short)0;
        }
      }
#pragma unroll
      for (int j = 0; j < 8; ++j)
        *reinterpret_cast<unsigned short*>(dst + fztc::kmajor_offset(8 * c + j, kk, TC_NKC)) = e[j];
    }
  }
}

template <int MODE, int EPI>
__global__ void __launch_bounds__(256, 1) k_gemm_tc(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda,
                                                    const __nv_bfloat16* __restrict__ B, int ldb,
                                                    const float* __restrict__ bias, const float* __restrict__ zin,
                                                    float* __restrict__ zout, float* __restrict__ fout,
                                                    __nv_bfloat16* __restrict__ out, int ldc, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  __shared__ __align__(8) uint64_t mbar[TC_STAGES];
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * 128, n0 = blockIdx.x * 128;
  // A: NT, NN K-contiguous rows of a (M x K); TN the transpose.  B: NT
  // K-contiguous rows of b (N x K); NN, TN the transpose.
  const bool akc = MODE != TN, bkc = MODE == NT;
  const bool avec = (lda % 8) == 0 && (((uintptr_t)A) & 15) == 0;
  const bool bvec = (ldb % 8) == 0 && (((uintptr_t)B) & 15) == 0;
  if (warp == 0) {
    fztc::tmem_alloc(&tbase, 128);
    fztc::tmem_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i < TC_STAGES; ++i) fztc::mbar_init(&mbar[i], 1);
    fztc::fence_mbar_init();
  }
  fztc::fence_before_sync();
  __syncthreads();
  fztc::fence_after_sync();
  const uint32_t tmem = tbase;
  const uint32_t idesc = fztc::idesc_bf16(128, 128);
  const int nkb = (K + TC_BK - 1) / TC_BK;
  bool ok = true;
  for (int kb = 0; kb < nkb && ok; ++kb) {
    const int buf = kb % TC_STAGES;
    unsigned char* as = tsm + (size_t)buf * 2 * TC_TILE;
    unsigned char* bs = as + TC_TILE;
    if (kb >= TC_STAGES) ok = fztc::mbar_wait(&mbar[buf], ((kb - TC_STAGES) / TC_STAGES) & 1, TC_WAIT_NS);
    ok = __syncthreads_and(ok);
    if (!ok) break;
    tc_stage(A, lda, akc, avec, m0, kb * TC_BK, M, K, as);
    tc_stage(B, ldb, bkc, bvec, n0, kb * TC_BK, N, K, bs);
    fztc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      const uint32_t sa = fztc::smem_addr(as), sb = fztc::smem_addr(bs);
#pragma unroll
      for (int ks = 0; ks < TC_BK / 16; ++ks) {
        const uint64_t da = fztc::desc_kmajor(sa + ks * 256, 128, TC_NKC * 128);
        const uint64_t db = fztc::desc_kmajor(sb + ks * 256, 128, TC_NKC * 128);
        fztc::mma_bf16(tmem, da, db, idesc, (kb > 0 || ks > 0) ? 1u : 0u);
      }
      fztc::commit(&mbar[buf]);
    }
  }
  if (ok && nkb > 0) {
    const int last = nkb - 1;
    ok = fztc::mbar_wait(&mbar[last % TC_STAGES], (last / TC_STAGES) & 1, TC_WAIT_NS);
  }
  ok = __syncthreads_and(ok);
  fztc::fence_after_sync();
  if (ok) {
    const int q = warp & 3, half = warp >> 2;
    const int m = m0 + 32 * q + lane;
#pragma unroll 1
    for (int cc = 0; cc < 64; cc += 16) {
      float v[16];
      fztc::tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(64 * half + cc), v);
      if (m >= M) continue;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int n = n0 + 64 * half + cc + i;
        if (n >= N) continue;
        const float c = v[i];
        const size_t o = (size_t)m * ldc + n;
        if (EPI == EPI_FWD_GELU) {
          const float z = c + bias[n];
          if (zout) zout[o] = z;
          out[o] = __float2bfloat16_rn(gelu(z));
        } else if (EPI == EPI_FWD_LIN) {
          fout[o] = c + bias[n];
        } else if (EPI == EPI_BWD_GELU) {
          out[o] = __float2bfloat16_rn(c * gelu_d(zin[o]));
        } else {
          fout[o] = c;
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  fztc::fence_before_sync();
  __syncthreads();
  if (warp == 0) fztc::tmem_dealloc(tmem, 128);
}

// The GEMMs whose bf16 operands sit in device memory with a 16-byte row
// stride, fed by the tensor memory accelerator: a 128 x 128 output tile per
// CTA of 256 threads, two CTAs per SM, K in blocks of 64 through three
// shared-memory stages.  An operand is K-major (AMN / BMN false: K
// contiguous, the forward's X and W) or MN-major (true: MN contiguous, the
// backward's dZ^T, X^T and W^T), the tensor core reading either layout.
// Warp 0's lane 0 issues the bulk tensor copies of A (128 x 64) and B
// (128 x 64) into a stage, 128-byte swizzled, and arms the stage's "full"
// mbarrier with their byte count; warp 1's lane 0 waits for it, issues the
// four tcgen05.mma of the block (FP32 accumulator in 128 TMEM columns) and
// commits them to the stage's "empty" mbarrier, which hands the stage back
// to the copies; the last commit arrives on "done".  Then all eight warps
// read the accumulator back (tcgen05.ld; warp w: TMEM lanes 32 (w % 4), 64
// columns from 64 (w / 4)) and apply the epilogue, 16-byte stores where the
// row stride allows.  Every wait is bounded (2 s): one that runs out sets
// the error flag and the CTA frees its tensor memory.
constexpr int TM_BM = 128, TM_BN = 128, TM_BK = 64, TM_ST = 3;
constexpr int TM_TILE_A = TM_BM * TM_BK * 2, TM_TILE_B = TM_BN * TM_BK * 2;   // 16 KB each
constexpr size_t TM_SMEM = (size_t)TM_ST * (TM_TILE_A + TM_TILE_B) + 1024;    // + the 1 KB alignment

template <int EPI, bool AMN, bool BMN>
__global__ void __launch_bounds__(256, 2) k_gemm_tma(const __grid_constant__ CUtensorMap ta,
                                                     const __grid_constant__ CUtensorMap tb, int M, int N, int K,
                                                     const float* __restrict__ bias, const float* __restrict__ zin,
                                                     float* __restrict__ zout, float* __restrict__ fout,
                                                     __nv_bfloat16* __restrict__ out, int ldc,
                                                     int* __restrict__ err) {
  extern __shared__ unsigned char tm_raw[];
  __shared__ __align__(8) uint64_t full[TM_ST], empty[TM_ST], done;
  __shared__ uint32_t tbase;
  __shared__ int bad;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * TM_BM, n0 = blockIdx.x * TM_BN;
  // the swizzled tiles start on a 1 KB boundary
  const uint32_t raw = fztc::smem_addr(tm_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* tiles = tm_raw + (base - raw);
  if (warp == 0) {
    fztc::tmem_alloc(&tbase, TM_BN);
    fztc::tmem_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i < TM_ST; ++i) {
      fztc::mbar_init(&full[i], 1);
      fztc::mbar_init(&empty[i], 1);
    }
    fztc::mbar_init(&done, 1);
    bad = 0;
    fztc::fence_mbar_init();
  }
  fztc::fence_before_sync();
  __syncthreads();
  fztc::fence_after_sync();
  const uint32_t tmem = tbase;
  const int nkb = (K + TM_BK - 1) / TM_BK;
  if (warp == 0) {
    if (lane == 0) {
      for (int kb = 0; kb < nkb; ++kb) {
        const int st = kb % TM_ST;
        // the stage's previous use (block kb - TM_ST) must have been consumed
        if (kb >= TM_ST && !fztc::mbar_wait(&empty[st], ((kb / TM_ST) - 1) & 1, TC_WAIT_NS)) {
          atomicExch(&bad, 1);
          break;
        }
        unsigned char* sa = tiles + (size_t)st * (TM_TILE_A + TM_TILE_B);
        unsigned char* sb = sa + TM_TILE_A;
        fztc::mbar_arrive_expect_tx(&full[st], TM_TILE_A + TM_TILE_B);
        // K-major: one 64 (K) x 128 box; MN-major: two 64 (MN) x 64 (K)
        // boxes, the second 64 MN elements 8 KB on
        if (AMN) {
          fztc::tma_load_2d(sa, &ta, m0, kb * TM_BK, &full[st]);
          fztc::tma_load_2d(sa + TM_TILE_A / 2, &ta, m0 + 64, kb * TM_BK, &full[st]);
        } else {
          fztc::tma_load_2d(sa, &ta, kb * TM_BK, m0, &full[st]);
        }
        if (BMN) {
          fztc::tma_load_2d(sb, &tb, n0, kb * TM_BK, &full[st]);
          fztc::tma_load_2d(sb + TM_TILE_B / 2, &tb, n0 + 64, kb * TM_BK, &full[st]);
        } else {
          fztc::tma_load_2d(sb, &tb, kb * TM_BK, n0, &full[st]);
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = fztc::idesc_bf16_major(TM_BM, TM_BN, AMN, BMN);
      int kb = 0;
      for (; kb < nkb; ++kb) {
        const int st = kb % TM_ST;
        if (!fztc::mbar_wait(&full[st], (kb / TM_ST) & 1, TC_WAIT_NS)) {
          atomicExch(&bad, 1);
          break;
        }
        fztc::fence_after_sync();
        const uint32_t sa = base + (uint32_t)st * (TM_TILE_A + TM_TILE_B), sb = sa + TM_TILE_A;
#pragma unroll
        for (int ks = 0; ks < TM_BK / 16; ++ks) {
          const uint64_t da = AMN ? fztc::desc_sw128_mn(sa + 2048 * ks, TM_TILE_A / 2) : fztc::desc_sw128(sa + 32 * ks);
          const uint64_t db = BMN ? fztc::desc_sw128_mn(sb + 2048 * ks, TM_TILE_B / 2) : fztc::desc_sw128(sb + 32 * ks);
          fztc::mma_bf16(tmem, da, db, idesc, (kb > 0 || ks > 0) ? 1u : 0u);
        }
        fztc::commit(&empty[st]);
      }
      if (kb == nkb) fztc::commit(&done);
    }
    __syncwarp();
  }
  bool ok = fztc::mbar_wait(&done, 0, TC_WAIT_NS);
  ok = __syncthreads_and(ok) && !*(volatile int*)&bad;
  fztc::fence_after_sync();
  if (ok) {
    const int q = warp & 3, half = warp >> 2;
    const int m = m0 + 32 * q + lane;
    const bool vec = (ldc & 7) == 0;
#pragma unroll 1
    for (int cc = 0; cc < 64; cc += 16) {
      float v[16];
      fztc::tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(64 * half + cc), v);
      if (m >= M) continue;
      const int nb = n0 + 64 * half + cc;
      const size_t o = (size_t)m * ldc + nb;
      if (vec && nb + 16 <= N) {
        if (EPI == EPI_FWD_GELU || EPI == EPI_FWD_LIN)
#pragma unroll
          for (int i = 0; i < 16; ++i) v[i] += __ldg(&bias[nb + i]);
        if (EPI == EPI_BWD_GELU) {
          uint32_t h[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float2 z = __ldg(reinterpret_cast<const float2*>(zin + o) + i);
            const __nv_bfloat162 t = __floats2bfloat162_rn(v[2 * i] * gelu_d(z.x), v[2 * i + 1] * gelu_d(z.y));
            h[i] = *reinterpret_cast<const uint32_t*>(&t);
          }
          *reinterpret_cast<uint4*>(out + o) = make_uint4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<uint4*>(out + o + 8) = make_uint4(h[4], h[5], h[6], h[7]);
        } else if (EPI == EPI_FWD_GELU) {
          if (zout)
#pragma unroll
            for (int i = 0; i < 16; i += 4)
              *reinterpret_cast<float4*>(zout + o + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
          uint32_t h[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const __nv_bfloat162 t = __floats2bfloat162_rn(gelu(v[2 * i]), gelu(v[2 * i + 1]));
            h[i] = *reinterpret_cast<const uint32_t*>(&t);
          }
          *reinterpret_cast<uint4*>(out + o) = make_uint4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<uint4*>(out + o + 8) = make_uint4(h[4], h[5], h[6], h[7]);
        } else {
#pragma unroll
          for (int i = 0; i < 16; i += 4)
            *reinterpret_cast<float4*>(fout + o + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
        }
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int n = nb + i;
          if (n >= N) continue;
          if (EPI == EPI_BWD_GELU) {
            out[o + i] = __float2bfloat16_rn(v[i] * gelu_d(zin[o + i]));
          } else if (EPI == EPI_F32) {
            fout[o + i] = v[i];
          } else {
            const float z = v[i] + bias[n];
            if (EPI == EPI_FWD_GELU) {
              if (zout) zout[o + i] = z;
              out[o + i] = __float2bfloat16_rn(gelu(z));
            } else {
              fout[o + i] = z;
            }
          }
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  fztc::fence_before_sync();
  __syncthreads();
  if (warp == 0) fztc::tmem_dealloc(tmem, TM_BN);
}

// Training-step state on the device, so that one captured step replays for
// every batch: the position in the epoch's batch order and the Adam step.
struct TrainState {
  int bi;
  int step;
};

// Row offset of the current batch (order: the epoch's batch permutation).
__device__ __forceinline__ size_t batch_row(const int* order, const TrainState* st, int n) {
  return order ? (size_t)order[st->bi] * n : 0;
}

// MSE loss 1/(n*nout) sum lw_j (y - t)^2 (lw: per-output weights, null =
// all 1) and dL/dy in bf16
__global__ void k_mse(int n, int nout, const float* __restrict__ y, const float* __restrict__ t,
                      __nv_bfloat16* __restrict__ dy, float* __restrict__ loss, const int* __restrict__ order,
                      const TrainState* __restrict__ st, const float* __restrict__ lw = nullptr) {
  __shared__ float red[8];
  t += batch_row(order, st, n) * nout;
  const size_t total = (size_t)n * nout;
  float s = 0.0f;
  const float sc = 2.0f / (float)total;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const float d = y[i] - t[i];
    const float wd = lw ? lw[i % nout] * d : d;
    s += wd * d;
    dy[i] = __float2bfloat16_rn(sc * wd);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float b = 0.0f;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) b += red[i];
    atomicAdd(loss, b / (float)total);
  }
}

// bias gradient: column sums of dZ (bf16, n x m)
__global__ void k_colsum(int n, int m, const __nv_bfloat16* __restrict__ dz, float* __restrict__ db) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  float s = 0.0f;
  for (int i = 0; i < n; ++i) s += __bfloat162float(dz[(size_t)i * m + j]);
  db[j] = s;
}

__global__ void k_to_bf16(size_t n, const float* __restrict__ x, __nv_bfloat16* __restrict__ y) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

// Observed Stokes rows (n x d, FP64, GAIN-normalised) standardised with the
// training set's mean and spread, (x - mu) / sd in FP32, as bf16 inputs.
__global__ void k_obs_bf16(size_t n, int d, const double* __restrict__ x, const float* __restrict__ mu,
                           const float* __restrict__ sd, __nv_bfloat16* __restrict__ y) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(i % d);
    y[i] = __float2bfloat16_rn(((float)x[i] - mu[f]) / sd[f]);
  }
}

// the current batch's rows (n x d) of x as bf16
__global__ void k_batch_bf16(int n, int d, const float* __restrict__ x, const int* __restrict__ order,
                             const TrainState* __restrict__ st, __nv_bfloat16* __restrict__ y) {
  x += batch_row(order, st, n) * d;
  const size_t total = (size_t)n * d;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

__global__ void k_train_advance(TrainState* st) {
  st->bi += 1;
  st->step += 1;
}

// Adam (Kingma & Ba 2015) on FP32 masters, refreshing the bf16 copy; the
// bias corrections 1/(1 - b^t) of step t = st->step + 1
__global__ void k_adam(size_t n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, __nv_bfloat16* __restrict__ wb, float lr, float b1, float b2,
                       const TrainState* __restrict__ st, float eps) {
  const float t = (float)(st->step + 1);
  const float c1 = 1.0f / (1.0f - powf(b1, t)), c2 = 1.0f / (1.0f - powf(b2, t));
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float wi = w[i] - lr * (a * c1) / (sqrtf(b * c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

// deterministic initial weights: uniform(-1,1)*sqrt(6/(fan_in+fan_out)) from a
// counter-based hash (splitmix64)
__global__ void k_init(size_t n, float* __restrict__ w, unsigned long long seed, float scale) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const float u = (float)((z >> 40) * (1.0 / 16777216.0)) * 2.0f - 1.0f;
    w[i] = u * scale;
  }
}

}  // namespace

struct fz_mlp {
  int device = 0;
  int nl = 0;                 // layers
  int dim[MLP_MAXL + 1] = {};
  // per layer: FP32 master W (out x in) and b, bf16 W, grads, Adam moments
  float *W[MLP_MAXL] = {}, *b[MLP_MAXL] = {}, *gW[MLP_MAXL] = {}, *gb[MLP_MAXL] = {};
  float *mW[MLP_MAXL] = {}, *vW[MLP_MAXL] = {}, *mb[MLP_MAXL] = {}, *vb[MLP_MAXL] = {};
  __nv_bfloat16* Wb[MLP_MAXL] = {};
  // activations for a batch capacity
  int cap = 0;
  __nv_bfloat16* act[MLP_MAXL + 1] = {};   // act[0] = input (bf16), act[l] = gelu(z_l)
  float* z[MLP_MAXL] = {};                 // pre-activations
  float* yout = nullptr;                    // last layer output (fp32)
  __nv_bfloat16* dz[MLP_MAXL] = {};        // dL/dz per layer
  float* loss = nullptr;
  long long step = 0;
  cudaStream_t stream = nullptr;
  TrainState* tstate = nullptr;   // device
  int* order = nullptr;           // device batch order of one epoch
  int order_cap = 0;
  int* d_err = nullptr;           // set by a tensor-core GEMM that gave up waiting for its MMAs
  float* d_lw = nullptr;          // per-output loss weights (null: all 1)
};

namespace {

int mlp_fail(cudaError_t e) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "fz_b200 mlp: CUDA error %s\n", cudaGetErrorString(e));
    return FZ_ERR_CUDA;
  }
  return 0;
}
#define MLP_CK(x)                 \
  do {                            \
    int _rc = mlp_fail(x);        \
    if (_rc) return _rc;          \
  } while (0)

int grid1(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

int mlp_reserve(fz_mlp* p, int n) {
  if (n <= p->cap) return 0;
  for (int l = 0; l <= p->nl; ++l) cudaFree(p->act[l]), p->act[l] = nullptr;
  for (int l = 0; l < p->nl; ++l) {
    cudaFree(p->z[l]), p->z[l] = nullptr;
    cudaFree(p->dz[l]), p->dz[l] = nullptr;
  }
  cudaFree(p->yout);
  p->yout = nullptr;
  p->cap = 0;
  for (int l = 0; l <= p->nl; ++l) MLP_CK(cudaMalloc(&p->act[l], (size_t)n * p->dim[l] * sizeof(__nv_bfloat16)));
  for (int l = 0; l < p->nl; ++l) {
    MLP_CK(cudaMalloc(&p->z[l], (size_t)n * p->dim[l + 1] * sizeof(float)));
    MLP_CK(cudaMalloc(&p->dz[l], (size_t)n * p->dim[l + 1] * sizeof(__nv_bfloat16)));
  }
  MLP_CK(cudaMalloc(&p->yout, (size_t)n * p->dim[p->nl] * sizeof(float)));
  p->cap = n;
  return 0;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// to the driver library); null when the driver does not provide it.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return EncodeTiledFn(nullptr);
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}

// A K-contiguous bf16 operand (rows x K, row stride ld elements) as a 2-D
// tensor map of 64 x 128 boxes with 128-byte swizzling.  False (the caller
// then stages the operand itself) when the operand has fewer rows than a
// box, or its base or row stride is not 16-byte aligned.
bool tmap_kmajor(CUtensorMap* m, const __nv_bfloat16* p, int rows, int K, int ld) {
  const EncodeTiledFn fn = encode_tiled();
  if (!fn || rows < TM_BM || K < TM_BK || (reinterpret_cast<uintptr_t>(p) & 15) || ((size_t)ld * 2) % 16) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)TM_BK, (cuuint32_t)TM_BM};
  const cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(p), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// An MN-contiguous bf16 operand (K rows of mn elements, row stride ld) as a
// 2-D tensor map of 64 x 64 boxes (MN inner) with 128-byte swizzling.
bool tmap_mnmajor(CUtensorMap* m, const __nv_bfloat16* p, int K, int mn, int ld) {
  const EncodeTiledFn fn = encode_tiled();
  if (!fn || mn < 64 || K < TM_BK || (reinterpret_cast<uintptr_t>(p) & 15) || ((size_t)ld * 2) % 16) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)mn, (cuuint64_t)K};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {64, (cuuint32_t)TM_BK};
  const cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(p), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int MODE, int EPI>
void gemm(cudaStream_t s, int* err, int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B,
          int ldb, const float* bias, const float* zin, float* zout, float* fout, __nv_bfloat16* out, int ldc) {
  const dim3 gtm((N + TM_BN - 1) / TM_BN, (M + TM_BM - 1) / TM_BM);
  CUtensorMap ma, mb;
  if constexpr (MODE == NT && (EPI == EPI_FWD_GELU || EPI == EPI_FWD_LIN)) {
    if (tmap_kmajor(&ma, A, M, K, lda) && tmap_kmajor(&mb, B, N, K, ldb)) {
      k_gemm_tma<EPI, false, false><<<gtm, 256, TM_SMEM, s>>>(ma, mb, M, N, K, bias, zin, zout, fout, out, ldc, err);
      return;
    }
  } else if constexpr (MODE == NN && EPI == EPI_BWD_GELU) {
    // A = dZ (M x K, K contiguous); B[n][k] = W[k][n]: W's rows are K
    if (tmap_kmajor(&ma, A, M, K, lda) && tmap_mnmajor(&mb, B, K, N, ldb) && (ldc & 7) == 0) {
      k_gemm_tma<EPI, false, true><<<gtm, 256, TM_SMEM, s>>>(ma, mb, M, N, K, bias, zin, zout, fout, out, ldc, err);
      return;
    }
  } else if constexpr (MODE == TN && EPI == EPI_F32) {
    // A[m][k] = dZ[k][m], B[n][k] = X[k][n]: both with K as the row index
    if (tmap_mnmajor(&ma, A, K, M, lda) && tmap_mnmajor(&mb, B, K, N, ldb)) {
      k_gemm_tma<EPI, true, true><<<gtm, 256, TM_SMEM, s>>>(ma, mb, M, N, K, bias, zin, zout, fout, out, ldc, err);
      return;
    }
  }
  const dim3 grid((N + 127) / 128, (M + 127) / 128);
  k_gemm_tc<MODE, EPI><<<grid, 256, TC_SMEM, s>>>(M, N, K, A, lda, B, ldb, bias, zin, zout, fout, out, ldc, err);
}

template <typename F>
cudaError_t tma_attrs(F* kernel) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TM_SMEM);
  return e == cudaSuccess ? cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100) : e;
}

// The tensor-core GEMMs' shared memory above the default 48 KB (set once,
// before any stream capture).
int gemm_tc_attrs() {
  cudaError_t e = cudaFuncSetAttribute(k_gemm_tc<NT, EPI_FWD_GELU>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)TC_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_gemm_tc<NT, EPI_FWD_LIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_gemm_tc<TN, EPI_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_gemm_tc<NN, EPI_BWD_GELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
  // two CTAs per SM (97 KB each): one CTA's epilogue overlaps the other's MMAs
  if (e == cudaSuccess) e = tma_attrs(k_gemm_tma<EPI_FWD_GELU, false, false>);
  if (e == cudaSuccess) e = tma_attrs(k_gemm_tma<EPI_FWD_LIN, false, false>);
  if (e == cudaSuccess) e = tma_attrs(k_gemm_tma<EPI_BWD_GELU, false, true>);
  if (e == cudaSuccess) e = tma_attrs(k_gemm_tma<EPI_F32, true, true>);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "fz_b200 mlp: CUDA error %s\n", cudaGetErrorString(e));
    return FZ_ERR_CUDA;
  }
  return 0;
}

// forward of n rows already in act[0]; output in yout; the pre-activations
// are kept for a backward pass only when keep_z
void mlp_fwd(fz_mlp* p, int n, bool keep_z = true) {
  for (int l = 0; l < p->nl; ++l) {
    const int in = p->dim[l], out = p->dim[l + 1];
    if (l + 1 < p->nl)
      gemm<NT, EPI_FWD_GELU>(p->stream, p->d_err, n, out, in, p->act[l], in, p->Wb[l], in, p->b[l], nullptr,
                             keep_z ? p->z[l] : nullptr, nullptr, p->act[l + 1], out);
    else
      gemm<NT, EPI_FWD_LIN>(p->stream, p->d_err, n, out, in, p->act[l], in, p->Wb[l], in, p->b[l], nullptr, nullptr, p->yout,
                            nullptr, out);
  }
}

// backward from dz[nl-1]; fills gW, gb
void mlp_bwd(fz_mlp* p, int n) {
  for (int l = p->nl - 1; l >= 0; --l) {
    const int in = p->dim[l], out = p->dim[l + 1];
    // dW (out x in) = dZ^T (out x n) X (n x in)
    gemm<TN, EPI_F32>(p->stream, p->d_err, out, in, n, p->dz[l], out, p->act[l], in, nullptr, nullptr, nullptr, p->gW[l],
                      nullptr, in);
    k_colsum<<<(out + 255) / 256, 256, 0, p->stream>>>(n, out, p->dz[l], p->gb[l]);
    if (l > 0)   // dZ_{l-1} = (dZ_l W_l) * gelu'(z_{l-1})
      gemm<NN, EPI_BWD_GELU>(p->stream, p->d_err, n, in, out, p->dz[l], out, p->Wb[l], in, nullptr, p->z[l - 1], nullptr,
                             nullptr, p->dz[l - 1], in);
  }
}

}  // namespace

extern "C" {

int fz_mlp_create(fz_mlp** out, int nlayers, const int* dims, unsigned long long seed, int device) {
  if (!out || nlayers < 1 || nlayers > MLP_MAXL || !dims) return FZ_ERR_ARG;
  for (int l = 0; l <= nlayers; ++l)
    if (dims[l] <= 0 || (l < nlayers && dims[l] % 8)) return FZ_ERR_ARG;   // input widths: 16-byte rows
  fz_mlp* p = new (std::nothrow) fz_mlp;
  if (!p) return FZ_ERR_NOMEM;
  p->device = device;
  p->nl = nlayers;
  for (int l = 0; l <= nlayers; ++l) p->dim[l] = dims[l];
  int rc = 0;
  auto fail = [&](int code) {
    fz_mlp_destroy(p);
    return code;
  };
  if ((rc = mlp_fail(cudaSetDevice(device)))) return fail(rc);
  if ((rc = mlp_fail(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking)))) return fail(rc);
  for (int l = 0; l < nlayers; ++l) {
    const size_t nw = (size_t)dims[l] * dims[l + 1];
    float** f32[] = {&p->W[l], &p->gW[l], &p->mW[l], &p->vW[l]};
    for (float** q : f32)
      if ((rc = mlp_fail(cudaMalloc(q, nw * sizeof(float))))) return fail(rc);
    float** f32b[] = {&p->b[l], &p->gb[l], &p->mb[l], &p->vb[l]};
    for (float** q : f32b)
      if ((rc = mlp_fail(cudaMalloc(q, dims[l + 1] * sizeof(float))))) return fail(rc);
    if ((rc = mlp_fail(cudaMalloc(&p->Wb[l], nw * sizeof(__nv_bfloat16))))) return fail(rc);
    const float sc = std::sqrt(6.0f / (float)(dims[l] + dims[l + 1]));
    k_init<<<grid1(nw), 256, 0, p->stream>>>(nw, p->W[l], seed + 1000003ull * l, sc);
    k_to_bf16<<<grid1(nw), 256, 0, p->stream>>>(nw, p->W[l], p->Wb[l]);
    cudaMemsetAsync(p->b[l], 0, dims[l + 1] * sizeof(float), p->stream);
    cudaMemsetAsync(p->mW[l], 0, nw * sizeof(float), p->stream);
    cudaMemsetAsync(p->vW[l], 0, nw * sizeof(float), p->stream);
    cudaMemsetAsync(p->mb[l], 0, dims[l + 1] * sizeof(float), p->stream);
    cudaMemsetAsync(p->vb[l], 0, dims[l + 1] * sizeof(float), p->stream);
  }
  if ((rc = mlp_fail(cudaMalloc(&p->loss, sizeof(float))))) return fail(rc);
  if ((rc = mlp_fail(cudaMalloc(&p->d_err, sizeof(int))))) return fail(rc);
  if ((rc = mlp_fail(cudaMemsetAsync(p->d_err, 0, sizeof(int), p->stream)))) return fail(rc);
  if ((rc = gemm_tc_attrs())) return fail(rc);
  if ((rc = mlp_fail(cudaStreamSynchronize(p->stream)))) return fail(rc);
  *out = p;
  return 0;
}

namespace {
// FZ_ERR_CUDA when a tensor-core GEMM of p gave up waiting (after the stream
// has completed); the flag is cleared.
int mlp_tc_status(fz_mlp* p) {
  int e = 0;
  if (mlp_fail(cudaMemcpy(&e, p->d_err, sizeof(int), cudaMemcpyDeviceToHost))) return FZ_ERR_CUDA;
  if (!e) return 0;
  cudaMemset(p->d_err, 0, sizeof(int));
  std::fprintf(stderr, "fz_b200 mlp: a tensor-core GEMM gave up waiting for its MMAs\n");
  return FZ_ERR_CUDA;
}
}  // namespace

int fz_mlp_destroy(fz_mlp* p) {
  if (!p) return 0;
  cudaSetDevice(p->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  for (int l = 0; l < MLP_MAXL; ++l) {
    cudaFree(p->W[l]);
    cudaFree(p->b[l]);
    cudaFree(p->gW[l]);
    cudaFree(p->gb[l]);
    cudaFree(p->mW[l]);
    cudaFree(p->vW[l]);
    cudaFree(p->mb[l]);
    cudaFree(p->vb[l]);
    cudaFree(p->Wb[l]);
    cudaFree(p->z[l]);
    cudaFree(p->dz[l]);
  }
  for (int l = 0; l <= MLP_MAXL; ++l) cudaFree(p->act[l]);
  cudaFree(p->yout);
  cudaFree(p->loss);
  cudaFree(p->d_err);
  cudaFree(p->d_lw);
  cudaFree(p->tstate);
  cudaFree(p->order);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
  return 0;
}

// Parameters as FP32 in layer order: W0 (out x in), b0, W1, b1, ...
long long fz_mlp_nparams(const fz_mlp* p) {
  if (!p) return FZ_ERR_ARG;
  long long n = 0;
  for (int l = 0; l < p->nl; ++l) n += (long long)p->dim[l] * p->dim[l + 1] + p->dim[l + 1];
  return n;
}

int fz_mlp_get_params(fz_mlp* p, float* host, int grads) {
  if (!p || !host) return FZ_ERR_ARG;
  MLP_CK(cudaSetDevice(p->device));
  MLP_CK(cudaStreamSynchronize(p->stream));
  size_t o = 0;
  for (int l = 0; l < p->nl; ++l) {
    const size_t nw = (size_t)p->dim[l] * p->dim[l + 1];
    MLP_CK(cudaMemcpy(host + o, grads ? p->gW[l] : p->W[l], nw * sizeof(float), cudaMemcpyDeviceToHost));
    o += nw;
    MLP_CK(cudaMemcpy(host + o, grads ? p->gb[l] : p->b[l], p->dim[l + 1] * sizeof(float), cudaMemcpyDeviceToHost));
    o += p->dim[l + 1];
  }
  return 0;
}

int fz_mlp_set_params(fz_mlp* p, const float* host) {
  if (!p || !host) return FZ_ERR_ARG;
  MLP_CK(cudaSetDevice(p->device));
  size_t o = 0;
  for (int l = 0; l < p->nl; ++l) {
    const size_t nw = (size_t)p->dim[l] * p->dim[l + 1];
    MLP_CK(cudaMemcpy(p->W[l], host + o, nw * sizeof(float), cudaMemcpyHostToDevice));
    o += nw;
    MLP_CK(cudaMemcpy(p->b[l], host + o, p->dim[l + 1] * sizeof(float), cudaMemcpyHostToDevice));
    o += p->dim[l + 1];
    k_to_bf16<<<grid1(nw), 256, 0, p->stream>>>(nw, p->W[l], p->Wb[l]);
  }
  MLP_CK(cudaGetLastError());
  MLP_CK(cudaStreamSynchronize(p->stream));
  return 0;
}

// Forward on device rows x (n x dim0, fp32) -> y (n x dimL, fp32), in chunks.
int fz_mlp_forward_device(fz_mlp* p, int n, const float* d_x, float* d_y, void* stream) {
  if (!p || n <= 0 || !d_x || !d_y) return FZ_ERR_ARG;
  MLP_CK(cudaSetDevice(p->device));
  const int chunk = 16384;
  int rc = mlp_reserve(p, std::min(n, chunk));
  if (rc) return rc;
  cudaStream_t s = p->stream;
  cudaEvent_t ev;
  MLP_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  if (stream) {   // order after the caller's stream
    cudaEventRecord(ev, (cudaStream_t)stream);
    cudaStreamWaitEvent(s, ev, 0);
  }
  const int d0 = p->dim[0], dl = p->dim[p->nl];
  for (int i = 0; i < n; i += chunk) {
    const int m = std::min(chunk, n - i);
    k_to_bf16<<<grid1((size_t)m * d0), 256, 0, s>>>((size_t)m * d0, d_x + (size_t)i * d0, p->act[0]);
    mlp_fwd(p, m, false);
    cudaMemcpyAsync(d_y + (size_t)i * dl, p->yout, (size_t)m * dl * sizeof(float), cudaMemcpyDeviceToDevice, s);
  }
  cudaEventRecord(ev, s);
  if (stream) cudaStreamWaitEvent((cudaStream_t)stream, ev, 0);
  int r2 = mlp_fail(cudaGetLastError());
  if (!stream) {
    cudaStreamSynchronize(s);
    if (!r2) r2 = mlp_tc_status(p);
  }
  cudaEventDestroy(ev);
  return r2;
}

// Forward of observed Stokes rows: d_obs (n x dim0, FP64) standardised by
// d_mu, d_sd (dim0, FP32) on the way to bf16, then the network; y (n x
// dimL, FP32).  Enqueued after the work on `stream`, which waits for it.
int fz_mlp_forward_obs_device(fz_mlp* p, int n, const double* d_obs, const float* d_mu, const float* d_sd, float* d_y,
                              void* stream) {
  if (!p || n <= 0 || !d_obs || !d_mu || !d_sd || !d_y) return FZ_ERR_ARG;
  MLP_CK(cudaSetDevice(p->device));
  const int chunk = 16384;
  int rc = mlp_reserve(p, std::min(n, chunk));
  if (rc) return rc;
  cudaStream_t s = p->stream;
  cudaEvent_t ev;
  MLP_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaEventRecord(ev, (cudaStream_t)stream);
  cudaStreamWaitEvent(s, ev, 0);
  const int d0 = p->dim[0], dl = p->dim[p->nl];
  for (int i = 0; i < n; i += chunk) {
    const int m = std::min(chunk, n - i);
    k_obs_bf16<<<grid1((size_t)m * d0), 256, 0, s>>>((size_t)m * d0, d0, d_obs + (size_t)i * d0, d_mu, d_sd,
                                                      p->act[0]);
    mlp_fwd(p, m, false);
    cudaMemcpyAsync(d_y + (size_t)i * dl, p->yout, (size_t)m * dl * sizeof(float), cudaMemcpyDeviceToDevice, s);
  }
  cudaEventRecord(ev, s);
  cudaStreamWaitEvent((cudaStream_t)stream, ev, 0);
  const int r2 = mlp_fail(cudaGetLastError());
  cudaEventDestroy(ev);
  return r2;
}

// Per-output weights of the training loss (host, nout values), or none
// (w null: every output weighs 1).
int fz_mlp_set_loss_weights(fz_mlp* p, const float* w, int n) {
  if (!p) return FZ_ERR_ARG;
  if (w && n != p->dim[p->nl]) return FZ_ERR_ARG;
  MLP_CK(cudaSetDevice(p->device));
  if (p->stream) MLP_CK(cudaStreamSynchronize(p->stream));
  if (!w) {
    cudaFree(p->d_lw);
    p->d_lw = nullptr;
    return 0;
  }
  for (int j = 0; j < n; ++j)
    if (!(w[j] >= 0.0f) || !std::isfinite(w[j])) return FZ_ERR_ARG;
  if (!p->d_lw) MLP_CK(cudaMalloc(&p->d_lw, (size_t)n * sizeof(float)));
  MLP_CK(cudaMemcpy(p->d_lw, w, (size_t)n * sizeof(float), cudaMemcpyHostToDevice));
  return 0;
}

int fz_mlp_io(const fz_mlp* p, int* nin, int* nout) {
  if (!p) return FZ_ERR_ARG;
  if (nin) *nin = p->dim[0];
  if (nout) *nout = p->dim[p->nl];
  return 0;
}

// Loss and gradients of one batch (no update); loss to *loss (host).
int fz_mlp_grad_device(fz_mlp* p, int n, const float* d_x, const float* d_t, float* loss) {
  if (!p || n <= 0 || !d_x || !d_t) return FZ_ERR_ARG;
  MLP_CK(cudaSetDevice(p->device));
  int rc = mlp_reserve(p, n);
  if (rc) return rc;
  cudaStream_t s = p->stream;
  const int d0 = p->dim[0], dl = p->dim[p->nl];
  k_to_bf16<<<grid1((size_t)n * d0), 256, 0, s>>>((size_t)n * d0, d_x, p->act[0]);
  mlp_fwd(p, n);
  MLP_CK(cudaMemsetAsync(p->loss, 0, sizeof(float), s));
  k_mse<<<grid1((size_t)n * dl), 256, 0, s>>>(n, dl, p->yout, d_t, p->dz[p->nl - 1], p->loss, nullptr, nullptr,
                                              p->d_lw);
  mlp_bwd(p, n);
  MLP_CK(cudaGetLastError());
  if (loss) MLP_CK(cudaMemcpyAsync(loss, p->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
  MLP_CK(cudaStreamSynchronize(s));
  return mlp_tc_status(p);
}

// Mini-batch Adam training over n device rows for `epochs` passes (rows
// visited in a fixed permutation per epoch from `seed`); mean loss of the
// last epoch to *loss.
int fz_mlp_train_device(fz_mlp* p, int n, const float* d_x, const float* d_t, int batch, int epochs, float lr,
                        unsigned long long seed, float* loss) {
  if (!p || n <= 0 || !d_x || !d_t || batch <= 0 || epochs <= 0) return FZ_ERR_ARG;
  MLP_CK(cudaSetDevice(p->device));
  int rc = mlp_reserve(p, batch);
  if (rc) return rc;
  cudaStream_t s = p->stream;
  const int d0 = p->dim[0], dl = p->dim[p->nl];
  const int nb = n / batch;
  if (nb <= 0) return FZ_ERR_ARG;
  if (!p->tstate && (rc = mlp_fail(cudaMalloc(&p->tstate, sizeof(TrainState))))) return rc;
  if (nb > p->order_cap) {
    cudaFree(p->order);
    p->order = nullptr;
    p->order_cap = 0;
    if ((rc = mlp_fail(cudaMalloc(&p->order, nb * sizeof(int))))) return rc;
    p->order_cap = nb;
  }
  // One training step (batch gather, forward, loss, backward, Adam, state
  // advance) captured once as a CUDA graph and replayed for every batch: the
  // batch offset and the Adam step come from the device state.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  if ((rc = mlp_fail(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)))) return rc;
  {
    k_batch_bf16<<<grid1((size_t)batch * d0), 256, 0, s>>>(batch, d0, d_x, p->order, p->tstate, p->act[0]);
    mlp_fwd(p, batch);
    k_mse<<<grid1((size_t)batch * dl), 256, 0, s>>>(batch, dl, p->yout, d_t, p->dz[p->nl - 1], p->loss, p->order,
                                                   p->tstate, p->d_lw);
    mlp_bwd(p, batch);
    const float b1 = 0.9f, b2 = 0.999f;
    for (int l = 0; l < p->nl; ++l) {
      const size_t nw = (size_t)p->dim[l] * p->dim[l + 1];
      k_adam<<<grid1(nw), 256, 0, s>>>(nw, p->W[l], p->gW[l], p->mW[l], p->vW[l], p->Wb[l], lr, b1, b2, p->tstate,
                                       1e-8f);
      k_adam<<<grid1(p->dim[l + 1]), 256, 0, s>>>(p->dim[l + 1], p->b[l], p->gb[l], p->mb[l], p->vb[l], nullptr, lr,
                                                  b1, b2, p->tstate, 1e-8f);
    }
    k_train_advance<<<1, 1, 0, s>>>(p->tstate);
  }
  rc = mlp_fail(cudaStreamEndCapture(s, &graph));
  if (!rc) rc = mlp_fail(cudaGraphInstantiate(&exec, graph, 0));
  // batch order: a fixed random permutation of the batch indices per epoch
  std::vector<int> order(nb);
  unsigned long long st = seed | 1ull;
  float last = 0.0f;
  for (int e = 0; e < epochs && !rc; ++e) {
    for (int i = 0; i < nb; ++i) order[i] = i;
    for (int i = nb - 1; i > 0; --i) {
      st ^= st << 13;
      st ^= st >> 7;
      st ^= st << 17;
      const int j = (int)(st % (unsigned long long)(i + 1));
      std::swap(order[i], order[j]);
    }
    const TrainState ts{0, (int)p->step};
    rc = mlp_fail(cudaMemcpyAsync(p->order, order.data(), nb * sizeof(int), cudaMemcpyHostToDevice, s));
    if (!rc) rc = mlp_fail(cudaMemcpyAsync(p->tstate, &ts, sizeof(ts), cudaMemcpyHostToDevice, s));
    if (!rc) rc = mlp_fail(cudaMemsetAsync(p->loss, 0, sizeof(float), s));
    for (int bi = 0; bi < nb && !rc; ++bi) rc = mlp_fail(cudaGraphLaunch(exec, s));
    p->step += nb;
    float h = 0.0f;
    if (!rc) rc = mlp_fail(cudaMemcpyAsync(&h, p->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    if (!rc) rc = mlp_fail(cudaStreamSynchronize(s));
    last = h / (float)nb;
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (!rc) rc = mlp_fail(cudaGetLastError());
  if (!rc) rc = mlp_tc_status(p);
  if (loss) *loss = last;
  return rc;
}

}  // extern "C"
