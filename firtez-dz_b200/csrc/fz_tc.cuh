// tcgen05 (fifth-generation tensor core) primitives for sm_100a, included
// by fz_cuda.cu and fz_mlp.cu.
//
// The kernels that use them stage bf16 operands in shared memory themselves
// (they convert, scale and split FP32 data on the way, which a bulk copy
// cannot), in the canonical K-major layout without swizzle: 8-row x 16-byte
// "core matrices", element (r, k) of a tile at
//     (r % 8) * 16 + (r / 8) * SBO + (k % 8) * 2 + (k / 8) * LBO   bytes,
// LBO the step between core matrices adjacent in K, SBO between core
// matrices adjacent in M (or N).  One elected thread issues
// tcgen05.mma.cta_group::1.kind::f16 (A, B bf16, D FP32 in tensor memory)
// and tcgen05.commit to an mbarrier; the epilogue reads D back with
// tcgen05.ld.32x32b (warp q of a warpgroup owns TMEM lanes 32q..32q+31).
// Every wait on an mbarrier is bounded in time (globaltimer): a wait that
// runs out reports it to the caller, which records an error and frees its
// tensor memory instead of spinning on.
#pragma once
#include <cstdint>

namespace fztc {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (K-major, SWIZZLE_NONE, Blackwell
// version bit 46): start address, LBO and SBO in 16-byte units.
__host__ __device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// The same for a K-major tile written by a bulk tensor copy with 128-byte
// swizzling: rows of 64 bf16 (128 B), the 16-byte chunks of row r stored at
// chunk index ^ (r % 8), 8-row groups 1 KB apart (SBO), LBO unused; layout
// type SWIZZLE_128B (2) at bits 61-63.  The tile starts on a 1 KB boundary
// and the MMA's 16-wide K step advances the start address by 32 B.
__host__ __device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(1024u >> 4) << 32) | ((uint64_t)1 << 46) |
         ((uint64_t)2 << 61);
}

// The same swizzle for an MN-major tile (MN contiguous): 128-byte rows of 64
// MN elements, one row per K index; 8-row K groups 1 KB apart (SBO), the
// next 64 MN elements lbo bytes on (LBO).  The MMA's 16-wide K step
// advances the start address by 16 rows = 2 KB.
__host__ __device__ __forceinline__ uint64_t desc_sw128_mn(uint32_t saddr, uint32_t lbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)(1024u >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16: D FP32 (bit 4), A and B bf16 (bits
// 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// ... with A (bit 15) and / or B (bit 16) MN-major
__host__ __device__ constexpr uint32_t idesc_bf16_major(int M, int N, bool a_mn, bool b_mn) {
  return idesc_bf16(M, N) | (a_mn ? 1u << 15 : 0u) | (b_mn ? 1u << 16 : 0u);
}

// D (+)= A B^T on the tensor core, issued by one thread; acc = 0 overwrites D.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// The mbarrier arrives once every tcgen05 operation this thread issued so
// far has completed.
__device__ __forceinline__ void commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for the completion of the mbarrier phase of the given parity, at most
// limit_ns; false when the time runs out.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint64_t limit_ns) {
  const uint32_t a = smem_addr(mbar);
  const uint64_t t0 = globaltimer();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (globaltimer() - t0 > limit_ns) return false;
  }
}

// Arrive on the mbarrier and add tx bytes to the phase's expected count.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar)), "r"(bytes)
               : "memory");
}

// One box of a 2-D tiled tensor map (x = innermost coordinate, in elements)
// into shared memory, completing tx bytes on the mbarrier.  Loads only from
// this GPU's memory; no multicast.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_addr(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(smem_addr(mbar))
      : "memory");
}

// Generic-proxy shared-memory writes made visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Tensor-memory allocation (one whole warp executes each): ncols a power of
// two >= 32; the base address is written to shared memory at dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of the warp's 32 TMEM lanes (warp-wide), then
// the wait for the load.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (r, k) of a K-major tile of bf16 with nkc = K/8
// core-matrix columns per 8-row group: groups row-major, so LBO = 128 and
// SBO = nkc * 128 (the MMA's 16-wide K step advances the start by 256 B).
__host__ __device__ constexpr uint32_t kmajor_offset(int r, int k, int nkc) {
  return (uint32_t)(((r >> 3) * nkc + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

}  // namespace fztc
