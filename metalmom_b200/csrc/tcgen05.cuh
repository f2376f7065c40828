// 5th-generation tensor-core helpers (inline PTX, sm_100a): shared-memory
// matrix descriptors for the 128-byte-swizzle layouts, the kind::f16
// instruction descriptor, tcgen05.mma / commit / fences and tensor-memory
// loads.  Used by the DFT-as-GEMM kernels and the tensor-core frame kernel.
#pragma once
#include <stdint.h>

namespace mm {

// Byte offset of element (row r, k) of 16-bit values in a K-major tile with
// 128-byte rows and the 128-byte swizzle (16-byte chunk index XOR row % 8).
__host__ __device__ __forceinline__ uint32_t sw128(int r, int k) {
  return (uint32_t)r * 128u + ((uint32_t)(((k >> 3) ^ (r & 7))) << 4) + (uint32_t)(k & 7) * 2u;
}

// K-major operand, 128-byte swizzle: rows of 128 bytes, 8-row groups 1024
// bytes apart (stride byte offset), sm_100 descriptor version 1.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;            // leading byte offset (unused by swizzled K-major)
  d |= (uint64_t)(1024u >> 4) << 32;  // stride byte offset
  d |= (uint64_t)1u << 46;            // descriptor version
  d |= (uint64_t)2u << 61;            // 128-byte swizzle
  return d;
}

// MN-major operand, 128-byte swizzle: atoms of 64 16-bit values along M/N
// (128 bytes) x 8 rows along K (1024 bytes, chunk index XOR K-row % 8);
// `lbo` bytes between atoms along M/N, `sbo` bytes between atoms along K
// (groups of 8 K-rows), descriptor version 1.
__device__ __forceinline__ uint64_t desc_mn_sw128(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;
  return d;
}

// kind::f16 instruction descriptor: f32 accumulator, A and B both bf16
// (F16 false) or both fp16 (F16 true; one instruction never mixes the two),
// B K-major, A K-major (a_mn false) or MN-major (a_mn true), M = m, N = n.
template <bool F16>
__host__ __device__ constexpr uint32_t idesc_f16kind(int n, int m = 128, bool a_mn = false) {
  return (1u << 4) | (F16 ? 0u : (1u << 7) | (1u << 10)) | (a_mn ? (1u << 15) : 0u) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D (tensor memory) = A * B^T (+ D when acc != 0), one CTA.
__device__ __forceinline__ void umma_f16kind(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

// Arrive on `mbar` once every tcgen05.mma this thread issued has completed.
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive 32-bit columns of this warp's 32 tensor-memory lanes.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// 64 consecutive 32-bit columns of this warp's 32 lanes: four loads, one wait.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float *v) {
  uint32_t r[64];
#pragma unroll
  for (int q = 0; q < 4; q++)
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[16 * q + 0]), "=r"(r[16 * q + 1]), "=r"(r[16 * q + 2]), "=r"(r[16 * q + 3]), "=r"(r[16 * q + 4]),
          "=r"(r[16 * q + 5]), "=r"(r[16 * q + 6]), "=r"(r[16 * q + 7]), "=r"(r[16 * q + 8]), "=r"(r[16 * q + 9]),
          "=r"(r[16 * q + 10]), "=r"(r[16 * q + 11]), "=r"(r[16 * q + 12]), "=r"(r[16 * q + 13]),
          "=r"(r[16 * q + 14]), "=r"(r[16 * q + 15])
        : "r"(taddr + 16u * q));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 64; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace mm
