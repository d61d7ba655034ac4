// umma.cuh -- fifth-generation tensor core (tcgen05) building blocks for
// sm_100a: tensor-memory allocation, shared-memory operand descriptors,
// BF16 x BF16 -> FP32 MMA issue, completion through an mbarrier and
// tensor-memory loads.
//
// Operands are kept in the "K-major, no swizzle" canonical layout: an R x K
// BF16 tile is cut into 8-row x 8-element core matrices of 128 contiguous
// bytes (row r of a core matrix at byte 16 r); core matrices adjacent along
// the rows are SBO = 128 bytes apart and those adjacent along K are
// LBO = (R / 8) * 128 bytes apart, so byte offset(r, c) =
// (c / 8) * LBO + (r / 8) * 128 + (r % 8) * 16 + (c % 8) * 2.
// One MMA consumes K = 16 (two core matrices along K); the next K step
// starts 2 * LBO bytes further.
//
// The accumulator of an M = 128 MMA (cta_group::1) occupies tensor-memory
// lanes 0..127 (lane = row) and N consecutive 32-bit columns; warp w of the
// block may read only lanes 32 (w % 4) .. 32 (w % 4) + 31.
#pragma once

#include <cstdint>

namespace acob200 {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, c) of a K-major tile with `rows` rows.
__host__ __device__ constexpr uint32_t kmajor_offset(int r, int c, int rows) {
  return (uint32_t)((c >> 3) * (rows >> 3) * 128 + (r >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}
// Distance between the K chunks of a tile with `rows` rows.
__host__ __device__ constexpr uint32_t kmajor_lbo(int rows) { return (uint32_t)(rows >> 3) * 128u; }
__host__ __device__ constexpr uint32_t kmajor_bytes(int rows, int k) {
  return (uint32_t)rows * (uint32_t)k * 2u;
}

// Shared-memory matrix descriptor (sm_100 format): start address, leading
// byte offset (K direction) and stride byte offset (row direction), all in
// 16-byte units; version 1 at bits 46-47; base offset 0; layout type 0
// (no swizzle) at bits 61-63.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 accumulator,
// both operands K-major, dense: D format bits 4-5 = 1 (F32), A format bits
// 7-9 = 1 (BF16), B format bits 10-12 = 1 (BF16), N >> 3 at bits 17-22,
// M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive (once) on the mbarrier when every MMA issued so far by this thread
// has completed.
__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// Tensor-memory allocation: one full warp; the base address is written to
// shared memory.  ncols is a power of two in [32, 512].
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy shared-memory writes made visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 consecutive 32-bit columns of this thread's lane (warp-collective).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace umma
}  // namespace acob200
