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
// code of each patch; 160 patches x 4 codes = K 640), B[(patch, code)][n]
// holds the per-step increments, n = (step, sum, part): each float32
// increment split into three bf16 parts hi + mid + lo that add up to it
// exactly, so the products are exact and the FP32 accumulation sums the
// float32 increments (in the tensor core's order, not the patch order of
// the reference: the sums agree to about one float32 rounding).
//
// One CTA (4 warps) owns 128 pixels (M = 128) and one group of 8 steps
// (N = 8 x 4 sums x 3 parts = 96) at a time; K runs in chunks of 16 patches
// (64 columns): the A chunk is built in shared memory by the threads from
// the pixel's bit words, the B chunk is copied from global memory
// (cp.async, prefetched one chunk ahead), both in the no-swizzle K-major
// core-matrix layout; one thread issues 4 tcgen05.mma (kind::f16, BF16 x
// BF16 -> FP32 in TMEM, 128 columns) per chunk and commits them to the
// chunk's mbarrier; two stages rotate.  The epilogue reads the accumulator
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
constexpr int kPsK = 640;                         // 160 patches x 4 codes
constexpr int kPsChunkK = 64;                     // 16 patches per chunk
constexpr int kPsChunks = kPsK / kPsChunkK;       // 10
constexpr int kPsABytes = 128 * kPsChunkK * 2;    // 16 KB (4 K steps of 4 KB)
constexpr int kPsBBytes = kPsN * kPsChunkK * 2;   // 12 KB (4 K steps of 3 KB)
constexpr int kPsStageBytes = kPsABytes + kPsBBytes;

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
  uint32_t w[4] = {0u, 0u, 0u, 0u};
  if (code_a >= 0) w[code_a >> 1] |= 0x3F80u << ((code_a & 1) * 16);
  if (code_b >= 0) w[2 + (code_b >> 1)] |= 0x3F80u << ((code_b & 1) * 16);
  return make_uint4(w[0], w[1], w[2], w[3]);
}

__global__ void __launch_bounds__(128) patch_sums_tc_kernel(const uint32_t* __restrict__ bits, int64_t npix,
                                                            int n_patches, const __nv_bfloat16* __restrict__ W,
                                                            int n_groups, int n_t, float* __restrict__ sums,
                                                            int* __restrict__ err, int wait_limit) {
  // dynamic shared memory: two stages of [A chunk | B chunk]; 56 KB per CTA
  // keeps at most 4 CTAs on an SM, so their TMEM (128 columns each) fits
  extern __shared__ __align__(1024) uint8_t ps_smem[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  const uint32_t base = tc::smem_u32(ps_smem);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t p = (int64_t)blockIdx.x * 128 + tid;
  const bool live = p < npix;
  uint32_t sw[SW100_CUBE_WORDS], vw[SW100_CUBE_WORDS];
#pragma unroll
  for (int w = 0; w < SW100_CUBE_WORDS; ++w) {
    sw[w] = live ? bits[(size_t)w * npix + p] : 0u;
    vw[w] = live ? bits[(size_t)(SW100_CUBE_WORDS + w) * npix + p] : 0u;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(&tmem_base)),
                 "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    tc::mbar_init(tc::smem_u32(&mbar[0]), 1);
    tc::mbar_init(tc::smem_u32(&mbar[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = tc::instr_desc(128, kPsN);

  // B chunk i of the whole sequence (group i / kPsChunks, chunk i % kPsChunks)
  // into a stage: 96 rows x 64 columns = 768 16-byte pieces, 6 per thread
  auto load_b = [&](int i, int stage) {
    const uint32_t b_st = base + stage * kPsStageBytes + kPsABytes;
    const __nv_bfloat16* wg = W + (size_t)(i / kPsChunks) * kPsN * kPsK + (i % kPsChunks) * kPsChunkK;
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      const int j = tid + 128 * m;
      const int n = j >> 3, u = j & 7;
      cp_async16_ps(b_st + (u >> 1) * (kPsN * 32) + tc::core_off(n, u & 1), wg + (size_t)n * kPsK + u * 8);
    }
  };

  // Iteration it (chunk c of group g): A(it) is built in its stage while
  // the previous chunk's MMAs run, then B(it + 1) is prefetched into the
  // other stage once those MMAs are done, and B(it), prefetched one
  // iteration earlier, is waited for.  Commits complete in order, so the
  // wait on MMA(it - 1) also covers every earlier chunk.
  const int total = n_groups * kPsChunks;
  bool ok = true;
  int last_commit = -1;
  load_b(0, 0);
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int it = 0; it < total; ++it) {
    const int stage = it & 1, g = it / kPsChunks, c = it % kPsChunks;
    const uint32_t a_st = base + stage * kPsStageBytes, b_st = a_st + kPsABytes;
    // A(it): this pixel's row, 4 K steps of 4 patches (the stage's last
    // reader, MMA(it - 2), was waited for in the previous iteration)
#pragma unroll
    for (int s = 0; s < 4; ++s) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int qa = c * 16 + s * 4 + h * 2, qb = qa + 1;
        int ca = -1, cb = -1;
        if (live && qa < n_patches)
          ca = (int)((sw[qa >> 5] >> (qa & 31)) & 1u) * 2 + (int)((vw[qa >> 5] >> (qa & 31)) & 1u);
        if (live && qb < n_patches)
          cb = (int)((sw[qb >> 5] >> (qb & 31)) & 1u) * 2 + (int)((vw[qb >> 5] >> (qb & 31)) & 1u);
        st_shared_v4(a_st + s * 4096 + tc::core_off(tid, h), onehot_pair(ca, cb));
      }
    }
    // MMA(it - 1) read the other stage: wait for it before refilling that stage
    if (it >= 1) {
      const bool w = tc::mbar_wait(tc::smem_u32(&mbar[(it - 1) & 1]), ((it - 1) >> 1) & 1, wait_limit);
      ok = __syncthreads_and(w) != 0;
      if (!ok) break;
    }
    if (it + 1 < total) load_b(it + 1, stage ^ 1);
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 1;" ::: "memory");   // B(it) has landed
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int s = 0; s < 4; ++s) {
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
      const bool w = tc::mbar_wait(tc::smem_u32(&mbar[stage]), (it >> 1) & 1, wait_limit);
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
      drained = tc::mbar_wait(tc::smem_u32(&mbar[last_commit & 1]), (last_commit >> 1) & 1,
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
