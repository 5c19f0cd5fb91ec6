/*
 * tc05.cuh — the fifth-generation tensor-core primitives the learned recovery
 * guess and its training use: tensor-memory allocation, one-thread MMA issue of
 * kind::f16 (BF16 operands, FP32 accumulators in tensor memory), commit to an
 * mbarrier, waits with an iteration limit, and the tensor-memory loads of the
 * epilogue. sm_100a only.
 *
 * Operand tiles live in shared memory in the canonical K-major layout without
 * swizzle: a tile of R rows (R % 8 == 0) and K columns (K % 8 == 0) of BF16
 * stores element (r, k) at byte
 *     (k / 8) * (R * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
 * i.e. 8x8 "core matrices" of 128 contiguous bytes; the 8-row groups are 128 B
 * apart (the stride byte offset) and the 8-column chunks R * 16 B apart (the
 * leading byte offset). One MMA consumes K = 16, two chunks; the k-th MMA of a
 * chain starts 2 * k * R * 16 bytes into the tile.
 *
 * D = A * B^T with A (M x K) and B (N x K) both K-major, M = 128: row m of D is
 * tensor-memory lane m, column n is column base + n; warp w of the CTA reads
 * lanes 32 w .. 32 w + 31.
 */
#pragma once
#include <cstdint>

#ifndef FX_HD
#define FX_HD __host__ __device__ __forceinline__
#endif

namespace tc05 {

/* byte offset of element (r, k) of a canonical K-major BF16 tile of R rows */
FX_HD constexpr uint32_t kmaj_off(uint32_t R, uint32_t r, uint32_t k) {
  return (k >> 3) * (R * 16u) + (r >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

/* shared-memory matrix descriptor: start address, leading byte offset (between
 * the K chunks), stride byte offset (between 8-row groups), all >> 4; version 1
 * (sm_100); base offset 0; no swizzle */
FX_HD constexpr uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1u << 46);
}

/* descriptor of the k16-th K = 16 slice of a canonical tile of R rows at saddr */
FX_HD constexpr uint64_t tile_desc(uint32_t saddr, uint32_t R, uint32_t k16) {
  return smem_desc(saddr + k16 * 2u * R * 16u, R * 16u, 128u);
}

/* instruction descriptor of kind::f16: FP32 accumulate (bits 4-5 = 1), A and B
 * BF16 (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at
 * bits 17-22, M >> 4 at bits 24-28 */
FX_HD constexpr uint32_t idesc_bf16_f32(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

#if defined(__CUDACC__)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

/* ---- tensor memory: one full warp allocates and frees ---- */
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(smem_u32(dst_smem)), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
/* generic-proxy writes to shared memory made visible to the tensor core's reads */
__device__ __forceinline__ void fence_smem_to_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

/* ---- the MMA (issued by one thread) and its completion ---- */
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate) : "memory");
}
/* arrives once on the mbarrier when every MMA this thread issued before it has completed */
__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
/* waits for the phase with parity `parity` to complete; gives up after `limit`
 * polls and returns false (the caller records the failure and unwinds) */
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done) : "r"(a), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}

/* ---- tensor memory -> registers: this thread's lane, 16 consecutive FP32 columns.
 * The load completes asynchronously; the wait names the destination registers as
 * its operands so that no use of them is scheduled before it. ---- */
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15])
               :: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

#endif  /* __CUDACC__ */

}  // namespace tc05
