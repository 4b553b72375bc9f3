// The flux loop's dense 153-patch sums on the 5th-generation tensor cores.
//
// Reference: solweig_gpu/solweig.py:683-724 (Kside_veg_v2022a, cyl = 1,
// anisotropic sky: KsideD = sum_p diffsh[p] * lumChi[p] * anglIncC[p] *
// ster[p] and the anisotropic diffuse luminance sum) and :1514-1541
// (define_patch_characteristics: the sky longwave of the patches where
// sh == 1 and vegsh == 1, downward and sideways).
//
// Per pixel and step these four sums take every patch, each patch adding a
// per-step increment chosen by the pixel's (sh, vegsh) code.  Written as a
// matrix product: A[pixel][(patch, code)] is one-hot (1.0 at the pixel's
// code of each patch; 156 patches x 4 codes = K 624), B[(patch, code)][n]
// holds the per-step increments, n = (step, sum, part): each float32
// increment split into three bf16 parts hi + mid + lo that add up to it
// exactly, so the products are exact and the FP32 accumulation sums the
// float32 increments (in the tensor core's order, not the patch order of
// the reference: the sums agree to about one float32 rounding).
//
// One CTA (4 warps) owns 128 pixels (M = 128) and one group of 8 steps
// (N = 8 x 4 sums x 3 parts = 96) at a time; K runs in chunks of 12 patches
// (48 columns): the A chunk is built in shared memory by the threads from
// the pixel's bit words, the B chunk is copied from global memory
// (cp.async, prefetched one chunk ahead), both in the no-swizzle K-major
// core-matrix layout; one thread issues 3 tcgen05.mma (kind::f16, BF16 x
// BF16 -> FP32 in TMEM, 128 columns) per chunk and commits them to the
// chunk's mbarrier; three stages rotate, two chunks' MMAs in flight.  The epilogue reads the accumulator
// with tcgen05.ld (warp w owns TMEM lanes 32 w .. 32 w + 31 = its pixels),
// adds the three parts and writes sums[(step * 4 + sum) * npix + pixel].
// Every wait is bounded: on expiry the CTA stops issuing, drains what it
// issued, frees its TMEM and records an error.
#include <cstdint>
#include <cuda_bf16.h>

#include "sw_common.cuh"
#include "tc_common.cuh"

namespace sw100 {

constexpr int kPsSteps = 8;                       // steps per group
constexpr int kPsN = kPsSteps * 4 * 3;            // 96 accumulator columns
constexpr int kPsK = 624;                         // 156 patches x 4 codes
constexpr int kPsChunkK = 48;                     // 12 patches per chunk (3 K steps)
constexpr int kPsChunks = kPsK / kPsChunkK;       // 13
constexpr int kPsABytes = 128 * kPsChunkK * 2;    // 12 KB (3 K steps of 4 KB)
constexpr int kPsBBytes = kPsN * kPsChunkK * 2;   // 9 KB (3 K steps of 3 KB)
constexpr int kPsStageBytes = kPsABytes + kPsBBytes;
constexpr int kPsStages = 3;                      // stages of [A | B] chunks in flight

// B = the per-step increments in bf16 parts: W[g][n][k], n = (step in the
// group * 4 + sum) * 3 + part, k = patch * 4 + code (code = sh * 2 + vegsh).
// Sums: 0 diffuse Kside (day), 1 anisotropic luminance (day), 2 sky
// longwave down, 3 sky longwave side (code 3 only).  Zero past the last
// step or patch.
__global__ void patch_weights_kernel(const sw100_time_step* __restrict__ steps, int n_t,
                                     const sw100_patch_step* __restrict__ patch, int n_patches,
                                     __nv_bfloat16* __restrict__ W, int n_groups) {
  const int64_t total = (int64_t)n_groups * kPsN * kPsK;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % kPsK);
    const int n = (int)((i / kPsK) % kPsN);
    const int g = (int)(i / ((int64_t)kPsK * kPsN));
    const int t = g * kPsSteps + n / 12, sum = (n % 12) / 3, part = n % 3;
    const int q = k >> 2, code = k & 3;
    float w = 0.f;
    if (t < n_t && q < n_patches) {
      const sw100_patch_step& P = patch[(size_t)t * n_patches + q];
      const bool day = steps[t].is_day != 0;
      if (sum == 0) w = day ? P.kside_d[code] : 0.f;
      else if (sum == 1) w = day ? P.anilum[code] : 0.f;
      else if (code == 3) w = (sum == 2) ? P.ld_sky : P.ls_sky;
    }
    // w = hi + mid + lo exactly (each difference is exact in float32)
    const __nv_bfloat16 hi = __float2bfloat16_rn(w);
    const float r1 = w - __bfloat162float(hi);
    const __nv_bfloat16 mid = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(mid);
    W[i] = part == 0 ? hi : (part == 1 ? mid : __float2bfloat16_rn(r2));
  }
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint4 v) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
               : "memory");
}

__device__ __forceinline__ void cp_async16_ps(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

// one-hot bf16 codes of two patches (8 columns = one 16-byte core-matrix row)
__device__ __forceinline__ uint4 onehot_pair(int code_a, int code_b) {
  const unsigned long long a = code_a >= 0 ? 0x3F80ull << (16 * code_a) : 0ull;   // columns 0-3
  const unsigned long long b = code_b >= 0 ? 0x3F80ull << (16 * code_b) : 0ull;   // columns 4-7
  return make_uint4((uint32_t)a, (uint32_t)(a >> 32), (uint32_t)b, (uint32_t)(b >> 32));
}

// B chunk i of the whole sequence (group i / kPsChunks, chunk i % kPsChunks)
// into a stage: 96 rows x 48 columns = 576 16-byte pieces (6 per row)
__device__ __forceinline__ void ps_load_b(const __nv_bfloat16* __restrict__ W, uint32_t base, int tid, int i,
                                          int stage) {
  const uint32_t b_st = base + stage * kPsStageBytes + kPsABytes;
  const __nv_bfloat16* wg = W + (size_t)(i / kPsChunks) * kPsN * kPsK + (i % kPsChunks) * kPsChunkK;
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    const int j = tid + 128 * m;
    if (j < kPsN * 6) {
      const int n = j / 6, u = j % 6;
      cp_async16_ps(b_st + (u >> 1) * (kPsN * 32) + tc::core_off(n, u & 1), wg + (size_t)n * kPsK + u * 8);
    }
  }
}

__global__ void __launch_bounds__(128) patch_sums_tc_kernel(const uint32_t* __restrict__ bits, int64_t npix,
                                                            int n_patches, const __nv_bfloat16* __restrict__ W,
                                                            int n_groups, int n_t, float* __restrict__ sums,
                                                            int* __restrict__ err, int wait_limit) {
  // dynamic shared memory: three stages of [A chunk | B chunk] (63 KB): at
  // most 3 CTAs share an SM, so their TMEM (128 columns each) fits in the
  // SM's 512 columns
  extern __shared__ __align__(128) uint8_t ps_smem[];
  __shared__ __align__(8) uint64_t mbar[kPsStages];
  __shared__ uint32_t tmem_base;
  const uint32_t base = tc::smem_u32(ps_smem);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t p = (int64_t)blockIdx.x * 128 + tid;
  const bool live = p < npix;
  // the pixel's sh and vegsh bit words (patches 32 w .. 32 w + 31), as scalars
  static_assert(SW100_CUBE_WORDS == 5, "five 32-bit words per patch cube");
  const uint32_t* bp = bits + (live ? p : 0);
  const size_t np = (size_t)npix;
  const uint32_t s0 = live ? bp[0 * np] : 0u, s1 = live ? bp[1 * np] : 0u, s2 = live ? bp[2 * np] : 0u,
                 s3 = live ? bp[3 * np] : 0u, s4 = live ? bp[4 * np] : 0u;
  const uint32_t v0 = live ? bp[5 * np] : 0u, v1 = live ? bp[6 * np] : 0u, v2 = live ? bp[7 * np] : 0u,
                 v3 = live ? bp[8 * np] : 0u, v4 = live ? bp[9 * np] : 0u;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(&tmem_base)),
                 "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int k = 0; k < kPsStages; ++k) tc::mbar_init(tc::smem_u32(&mbar[k]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = tc::instr_desc(128, kPsN);


  // Iteration it (chunk c of group g) uses stage it % 3: A(it) is built
  // there (its last reader, MMA(it - 3), was waited for in the previous
  // iteration); then MMA(it - 2) is waited for and B(it + 1) prefetched
  // into its stage, and B(it), prefetched one iteration earlier, is waited
  // for, so MMA(it - 1) may still run while MMA(it) is issued.  Commits
  // complete in order: a wait on MMA(j) covers every earlier chunk.
  const int total = n_groups * kPsChunks;
  bool ok = true;
  int last_commit = -1;
  ps_load_b(W, base, tid, 0, 0);
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int it = 0; it < total; ++it) {
    const int stage = it % kPsStages, g = it / kPsChunks, c = it % kPsChunks;
    const uint32_t a_st = base + stage * kPsStageBytes, b_st = a_st + kPsABytes;
    // A(it): this pixel's row, 3 K steps of 4 patches (see above); the
    // chunk's 12 patch bits are taken from the two words holding them,
    // selected into registers (no dynamic indexing)
    const int q0 = c * 12, cw = q0 >> 5, sh = q0 & 31;
    const uint32_t sa = cw == 0 ? s0 : cw == 1 ? s1 : cw == 2 ? s2 : cw == 3 ? s3 : s4;
    const uint32_t sb = cw == 0 ? s1 : cw == 1 ? s2 : cw == 2 ? s3 : cw == 3 ? s4 : 0u;
    const uint32_t va = cw == 0 ? v0 : cw == 1 ? v1 : cw == 2 ? v2 : cw == 3 ? v3 : v4;
    const uint32_t vb = cw == 0 ? v1 : cw == 1 ? v2 : cw == 2 ? v3 : cw == 3 ? v4 : 0u;
    const uint32_t ws = (uint32_t)((((unsigned long long)sb << 32) | sa) >> sh);   // bits of patches q0 ..
    const uint32_t wv = (uint32_t)((((unsigned long long)vb << 32) | va) >> sh);
#pragma unroll
    for (int s = 0; s < 3; ++s) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int ja = s * 4 + h * 2, jb = ja + 1;
        const int ca = (live && q0 + ja < n_patches) ? (int)((ws >> ja) & 1u) * 2 + (int)((wv >> ja) & 1u) : -1;
        const int cb = (live && q0 + jb < n_patches) ? (int)((ws >> jb) & 1u) * 2 + (int)((wv >> jb) & 1u) : -1;
        st_shared_v4(a_st + s * 4096 + tc::core_off(tid, h), onehot_pair(ca, cb));
      }
    }
    // the stage of B(it + 1) was last read by MMA(it - 2)
    if (it >= 2) {
      const int j = it - 2;
      const bool w = tc::mbar_wait(tc::smem_u32(&mbar[j % kPsStages]), (j / kPsStages) & 1, wait_limit);
      ok = __syncthreads_and(w) != 0;
      if (!ok) break;
    }
    if (it + 1 < total) ps_load_b(W, base, tid, it + 1, (it + 1) % kPsStages);
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 1;" ::: "memory");   // B(it) has landed
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const uint64_t ad = tc::smem_desc(a_st + s * 4096, 128, 256);
        const uint64_t bd = tc::smem_desc(b_st + s * (kPsN * 32), 128, 256);
        tc::mma_f16(tmem, ad, bd, idesc, (c > 0 || s > 0) ? 1u : 0u);
      }
      tc::commit(tc::smem_u32(&mbar[stage]));
      last_commit = it;
    }
    if (c + 1 < kPsChunks) continue;
    // the group's last chunk: its commit covers every MMA of the group
    {
      const bool w = tc::mbar_wait(tc::smem_u32(&mbar[stage]), (it / kPsStages) & 1, wait_limit);
      ok = __syncthreads_and(w) != 0;
      if (!ok) break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // epilogue: 48 columns (16 step x sum entries) at a time
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      uint32_t v[48];
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(half * 48 + x * 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[x * 16 + 0]), "=r"(v[x * 16 + 1]), "=r"(v[x * 16 + 2]), "=r"(v[x * 16 + 3]),
              "=r"(v[x * 16 + 4]), "=r"(v[x * 16 + 5]), "=r"(v[x * 16 + 6]), "=r"(v[x * 16 + 7]),
              "=r"(v[x * 16 + 8]), "=r"(v[x * 16 + 9]), "=r"(v[x * 16 + 10]), "=r"(v[x * 16 + 11]),
              "=r"(v[x * 16 + 12]), "=r"(v[x * 16 + 13]), "=r"(v[x * 16 + 14]), "=r"(v[x * 16 + 15])
            : "r"(addr));
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int m = half * 16 + e;           // step in group * 4 + sum
        const int t = g * kPsSteps + (m >> 2);
        const float s3 = (__uint_as_float(v[3 * e]) + __uint_as_float(v[3 * e + 1])) + __uint_as_float(v[3 * e + 2]);
        if (live && t < n_t) sums[((size_t)t * 4 + (m & 3)) * npix + p] = s3;
      }
    }
    // the next group's MMAs overwrite the accumulator
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (!ok) {
    // drain: no copy left in flight; the MMAs issued so far (the last
    // commit covers them all) are waited for before their TMEM is freed
    asm volatile("cp.async.wait_all;" ::: "memory");
    bool drained = true;
    if (tid == 0 && last_commit >= 0)
      drained = tc::mbar_wait(tc::smem_u32(&mbar[last_commit % kPsStages]), (last_commit / kPsStages) & 1,
                              wait_limit > (1 << 22) ? wait_limit : (1 << 22));
    drained = __syncthreads_and(drained) != 0;
    if (tid == 0 && err) atomicExch(err, drained ? 1 : 2);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
}

}  // namespace sw100
