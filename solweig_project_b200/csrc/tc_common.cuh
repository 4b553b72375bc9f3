// tcgen05 helpers shared by the tensor-core kernels (the preview network's
// convolutions, nn.cu, and the flux loop's patch sums, patch_sums.cu):
// shared-memory addresses, bounded mbarrier waits, the no-swizzle K-major
// shared-memory matrix descriptor, the kind::f16 instruction descriptor
// (BF16 A and B, FP32 accumulator), the MMA issue and commit, and the
// core-matrix offset of a row in a 16-wide K tile.
#pragma once
#include <cstdint>

namespace sw100 {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait: at most `limit` polls; false when it gave up
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i)
    if (mbar_try_wait(addr, parity)) return true;
  return false;
}

// 64-bit shared-memory matrix descriptor: no swizzle, K-major, LBO / SBO in bytes
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M x N
__device__ __forceinline__ uint32_t instr_desc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

// core-matrix offset (bytes) of row r, K half h in a 16-wide K-major tile
__device__ __forceinline__ int core_off(int r, int h) { return (r >> 3) * 256 + h * 128 + (r & 7) * 16; }

}  // namespace tc

}  // namespace sw100
