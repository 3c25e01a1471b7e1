// Fifth-generation tensor cores (tcgen05) for the precision form's tile
// scoring: shared-memory matrix descriptors, the MMA and its completion
// barrier, tensor-memory allocation and loads, in inline PTX (sm_100a).
//
// Operands are K-major with no swizzle: the canonical layout of 8-row x
// 16-byte core matrices, element (row r, byte b) of an operand at
//   (r / 8) * SBO + (b / 16) * LBO + (r % 8) * 16 + b % 16,
// here with LBO = 128 (core matrices adjacent along K) and SBO = 128 x the
// 16-byte chunks of a row (8-row groups one after another). One MMA reads
// K = 32 bytes (two chunks): 16 bfloat16 or 32 FP8 values.
#pragma once
#include <cstdint>

namespace pann {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of (row r, 16-byte chunk c) in the core-matrix layout of rows of `chunks` chunks.
__host__ __device__ __forceinline__ uint32_t cm_offset(uint32_t r, uint32_t c, uint32_t chunks) {
  return (r >> 3) * (chunks * 128u) + c * 128u + (r & 7u) * 16u;
}

// Shared-memory matrix descriptor: start address, LBO and SBO in 16-byte
// units (bits 0-13, 16-29, 32-45), descriptor version 1 (bits 46-47), base
// offset 0, no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;
  return d;
}

// Instruction descriptor: float32 accumulator (bits 4-5 = 1), A and B
// formats (bits 7-9, 10-12), both K-major, N >> 3 (bits 17-22), M >> 4
// (bits 24-28). kind::f16 with bfloat16 operands: format 1; kind::f8f6f4
// with E4M3 operands: format 0.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t ab_format, uint32_t M, uint32_t N) {
  return (1u << 4) | (ab_format << 7) | (ab_format << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one K step, issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void umma_fp8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// Arrive once on the mbarrier when every MMA this thread issued has completed.
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for the phase with the given parity to complete; gives up (returns
// false) after `limit_ns` nanoseconds, so a lost arrival cannot hang the kernel.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint64_t limit_ns) {
  const uint64_t t0 = globaltimer_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
}

// Generic-proxy writes to shared memory (stores, cp.async) made visible to
// the tensor core's reads.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// Tensor-memory allocation of `ncols` columns (a power of two >= 32) by one
// whole warp; the address is written to shared memory at `slot`.
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Four consecutive accumulator columns of this thread's lane (warp w of the
// warpgroup reads lanes 32 w .. 32 w + 31), then wait for the load.
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float* v) {
  uint32_t a, b, c, d;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(a), "=r"(b), "=r"(c), "=r"(d)
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  v[0] = __uint_as_float(a);
  v[1] = __uint_as_float(b);
  v[2] = __uint_as_float(c);
  v[3] = __uint_as_float(d);
}

}  // namespace pann
