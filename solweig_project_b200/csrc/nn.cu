// Kernels of the learned SVF preview: a small U-Net in BF16 with FP32
// accumulation on the tensor cores (tcgen05.mma for the convolutions'
// forward and data-gradient passes, mma.sync m16n8k16 for the weight
// gradients), trained on the GPU by these forward and backward kernels.
//
// Layout: activations NHWC bf16 with a channel stride (a buffer may hold a
// concatenation: a layer reads / writes channels [coff, coff + C) of a
// buffer of `stride` channels); channel counts and offsets are multiples of
// 16.  3 x 3 convolution weights, same padding, tap t = 3 * (dy + 1) +
// (dx + 1):
//   forward layout  Wf[t][co][ci]  (bf16; ci contiguous)
//   data-grad layout Wd[8 - t][ci][co] (bf16; the flipped kernel with the
//                    channel roles swapped, so dgrad is a forward conv)
//   master / grads  float32 in the forward layout, bias float32[co].
//
// Convolutions are implicit GEMMs.  Forward and data gradient: tcgen05.mma
// (below).  Weight gradient: a block reduces 64 output channels (M) x 64
// input channels (N) over a run of pixels (K) with mma.sync; its tiles are
// staged in shared memory with rows padded to 48 bytes (conflict-free
// fragment loads).
#include <cstdint>
#include <cuda_bf16.h>

#include "sw_common.cuh"
#include "tc_common.cuh"

namespace sw100 {

constexpr int kPad = 24;     // bf16 per staged row of the weight-gradient tiles (16 used)

__device__ __forceinline__ uint32_t ld_smem_u32(const __nv_bfloat16* p) {
  return *reinterpret_cast<const uint32_t*>(p);
}

__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ------------------------------------------------- tcgen05 convolution
// The same 3 x 3 convolution on the 5th-generation tensor cores: one CTA
// (4 warps) owns 128 consecutive pixels of the flattened (n, h, w) index
// (M = 128) and every output channel (N = Cout, 16..128); K runs over
// (tap, 16 input channels).  A pipeline stage holds 4 K steps: per step the
// 128 x 16 A tile and the Cout x 16 B tile in the no-swizzle K-major
// core-matrix layout (8 rows x 16 bytes per core matrix; the two 8-element
// halves of K 128 bytes apart, row groups 256 bytes apart), filled by
// cp.async straight from global memory.  Three stages rotate: the copies of
// stage g + 2 run while the MMAs of stage g do; one thread issues
// the stage's tcgen05.mma (kind::f16, BF16 x BF16 -> FP32) into a TMEM
// accumulator and tcgen05.commit arrives on the stage's mbarrier when they
// have read it.  The epilogue reads the accumulator
// with tcgen05.ld (warp w owns TMEM lanes 32 w .. 32 w + 31 = its pixels).
// Every wait is bounded: on expiry the CTA records an error, stops issuing
// and still frees its TMEM.

// K steps of 16 per pipeline stage, the shared-memory bytes of a stage's A
// (and B) tiles, and the stages in flight
constexpr int kTcStepsPerStage = 4;
constexpr int kTcStageBytes = kTcStepsPerStage * 4096;
constexpr int kTcStages = 3;
// polls of an mbarrier before a wait gives up (the default wait limit)
constexpr int kTcWaitLimit = 1 << 22;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

__global__ void __launch_bounds__(128) nn_conv3x3_tc_kernel(const __nv_bfloat16* __restrict__ X, int N, int H, int W,
                                                            int Cin, int xstride, int xcoff,
                                                            const __nv_bfloat16* __restrict__ Wt,
                                                            const float* __restrict__ bias, int Cout, void* Yv,
                                                            int ystride, int ycoff, int relu, int out_f32,
                                                            int* __restrict__ err, int wait_limit) {
  // dynamic shared memory: kTcStages A stage buffers (128 pixels x 64 K),
  // then kTcStages B stage buffers sized by the output channels (Cout x 64
  // K), 1024-byte aligned: 60 KB for Cout <= 32, 72 KB for 64, 96 KB for
  // 128, so 3, 3 and 2 CTAs per SM, whose TMEM allocations (32, 64 and 128
  // columns each) never exceed the SM's 512 columns
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  __shared__ __align__(8) uint64_t mbar[kTcStages];
  __shared__ uint32_t tmem_base;
  const uint32_t a_base = tc::smem_u32(tc_smem);
  const uint32_t b_base = a_base + kTcStages * kTcStageBytes;
  const uint32_t b_step = 32u * (uint32_t)Cout;                   // one K step of B: Cout / 8 core matrices
  const uint32_t b_stage = kTcStepsPerStage * b_step;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t total = (int64_t)N * H * W;
  const int64_t p0 = (int64_t)blockIdx.x * 128;
  const int ncols = Cout <= 32 ? 32 : (Cout <= 64 ? 64 : 128);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(&tmem_base)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int k = 0; k < kTcStages; ++k) tc::mbar_init(tc::smem_u32(&mbar[k]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;

  // this thread's pixel (A row) and output channel (B row)
  const int64_t pix = p0 + tid;
  int n = 0, h = 0, w = 0;
  const bool live = pix < total;
  if (live) {
    w = (int)(pix % W);
    h = (int)((pix / W) % H);
    n = (int)(pix / ((int64_t)W * H));
  }
  const uint32_t idesc = tc::instr_desc(128, Cout);
  const int kchunks = Cin / 16;
  const int nsteps = 9 * kchunks;
  const int nstages = (nsteps + kTcStepsPerStage - 1) / kTcStepsPerStage;

  // asynchronous copies of stage g into its buffer (zero fill outside the image)
  auto load_stage = [&](int g) {
    const int buf = g % kTcStages;
    const int s0 = g * kTcStepsPerStage;
    const int ns = min(kTcStepsPerStage, nsteps - s0);
    for (int j = 0; j < ns; ++j) {
      const int s = s0 + j;
      const int t = s / kchunks, ci0 = (s % kchunks) * 16;
      const int hs = h + t / 3 - 1, ws = w + t % 3 - 1;
      const bool in = live && hs >= 0 && hs < H && ws >= 0 && ws < W;
      const __nv_bfloat16* src = in ? X + (((size_t)n * H + hs) * W + ws) * xstride + xcoff + ci0 : X;
      const uint32_t a = a_base + buf * kTcStageBytes + j * 4096;
      cp_async16(a + tc::core_off(tid, 0), src, in ? 16 : 0);
      cp_async16(a + tc::core_off(tid, 1), src + 8, in ? 16 : 0);
      if (tid < Cout) {
        const __nv_bfloat16* wsrc = Wt + ((size_t)t * Cout + tid) * Cin + ci0;
        const uint32_t b = b_base + buf * b_stage + j * b_step;
        cp_async16(b + tc::core_off(tid, 0), wsrc, 16);
        cp_async16(b + tc::core_off(tid, 1), wsrc + 8, 16);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };

  // Pipeline status, the same for every thread of the block (each wait's
  // outcome is combined with __syncthreads_and).  Once a wait has run out,
  // no further copy or MMA is issued: the block drains what it issued and
  // frees its tensor memory.
  bool ok = true;
  int last_commit = -1;  // the last stage whose MMAs were committed (thread 0)
  load_stage(0);
  if (nstages > 1) load_stage(1);
  for (int g = 0; g < nstages && ok; ++g) {
    const int buf = g % kTcStages;
    // this stage's copies are done (the next stage's may still be in flight)
    if (g + 1 < nstages) asm volatile("cp.async.wait_group 1;" ::: "memory");
    else asm volatile("cp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int s0 = g * kTcStepsPerStage;
      const int ns = min(kTcStepsPerStage, nsteps - s0);
      for (int j = 0; j < ns; ++j) {
        const uint64_t ad = tc::smem_desc(a_base + buf * kTcStageBytes + j * 4096, 128, 256);
        const uint64_t bd = tc::smem_desc(b_base + buf * b_stage + j * b_step, 128, 256);
        tc::mma_f16(tmem, ad, bd, idesc, (s0 + j) > 0 ? 1u : 0u);
      }
      tc::commit(tc::smem_u32(&mbar[buf]));
      last_commit = g;
    }
    // stage g + 2 reuses the buffer of stage g - 1: wait for its MMAs first
    if (g + 2 < nstages) {
      bool w = true;
      if (g >= 1) w = tc::mbar_wait(tc::smem_u32(&mbar[(g - 1) % kTcStages]), ((g - 1) / kTcStages) & 1, wait_limit);
      ok = __syncthreads_and(w) != 0;
      if (ok) load_stage(g + 2);
    }
  }
  // the last stage's MMAs (its commit covers every earlier one)
  if (ok && nstages > 0) {
    const bool w =
        tc::mbar_wait(tc::smem_u32(&mbar[(nstages - 1) % kTcStages]), ((nstages - 1) / kTcStages) & 1, wait_limit);
    ok = __syncthreads_and(w) != 0;
  }
  if (!ok) {
    // drain: no copy is left in flight, and the MMAs issued so far (the last
    // commit covers them all) are waited for with the default limit before
    // the tensor memory they write is freed
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    bool drained = true;
    if (tid == 0 && last_commit >= 0)
      drained = tc::mbar_wait(tc::smem_u32(&mbar[last_commit % kTcStages]), (last_commit / kTcStages) & 1,
                              max(wait_limit, kTcWaitLimit));
    drained = __syncthreads_and(drained) != 0;
    if (tid == 0 && err) atomicExch(err, drained ? 1 : 2);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // epilogue: 16 columns at a time from this warp's 32 TMEM lanes
  if (ok) {
    for (int c0 = 0; c0 < Cout; c0 += 16) {
      uint32_t v[16];
      const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(addr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (live) {
        const size_t o = (size_t)pix * ystride + ycoff + c0;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          float x = __uint_as_float(v[e]) + (bias ? bias[c0 + e] : 0.f);
          if (relu) x = fmaxf(x, 0.f);
          if (out_f32) reinterpret_cast<float*>(Yv)[o + e] = x;
          else reinterpret_cast<__nv_bfloat16*>(Yv)[o + e] = __float2bfloat16_rn(x);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// dW[t][co][ci] += sum_px dY[px, co] * X[px + (dy, dx), ci] over a chunk of
// pixels (one image row of 64 pixels per K step); dbias[co] += sum dY
// (tap 4 blocks only).  grid: (ceil(W / 64) * H * N / rows_per_block ... )
// organised as (row chunk, 9 taps, co tiles * ci tiles).  block 128: warp w
// owns output channels co0 + 16 w .. +15 (M) x 64 input channels (N).
__global__ void __launch_bounds__(128) nn_wgrad_kernel(const __nv_bfloat16* __restrict__ X, int N, int H, int W,
                                                       int Cin, int xstride, int xcoff,
                                                       const __nv_bfloat16* __restrict__ dY, int Cout, int dstride,
                                                       int dcoff, float* __restrict__ dW, float* __restrict__ dbias,
                                                       int rows_per_block) {
  __shared__ __align__(16) __nv_bfloat16 As[64][kPad];   // [co][px]
  __shared__ __align__(16) __nv_bfloat16 Bs[64][kPad];   // [ci][px]
  const int n_ci = (Cin + 63) / 64, n_co = (Cout + 63) / 64;
  const int t = blockIdx.y;
  const int co0 = (blockIdx.z / n_ci) * 64, ci0 = (blockIdx.z % n_ci) * 64;
  const int dy = t / 3 - 1, dx = t % 3 - 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, tq = lane & 3;
  const int n_wt = (W + 15) / 16;
  const int total_rows = N * H;
  float acc[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  float bsum = 0.f;
  (void)n_co;
  const int row_begin = blockIdx.x * rows_per_block;
  const int row_end = min(total_rows, row_begin + rows_per_block);
  for (int row = row_begin; row < row_end; ++row) {
    const int n = row / H, h = row % H;
    const int hs = h + dy;
    for (int wt = 0; wt < n_wt; ++wt) {
      const int w0 = wt * 16;
      // stage A[co][px]: 64 channels x 16 pixels of dY; thread: px = tid / 8, 8 channels (tid % 8) * 8
      {
        const int px = tid >> 3, c8 = (tid & 7) * 8;
        const int w = w0 + px;
        __nv_bfloat16 v[8];
        if (w < W && co0 + c8 < Cout) {
          const uint4 u = *reinterpret_cast<const uint4*>(dY + (((size_t)n * H + h) * W + w) * dstride + dcoff + co0 + c8);
          *reinterpret_cast<uint4*>(v) = u;
        } else {
#pragma unroll
          for (int e = 0; e < 8; ++e) v[e] = __float2bfloat16_rn(0.f);
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) As[c8 + e][px] = v[e];
      }
      // stage B[ci][px]: 64 input channels x 16 shifted pixels of X
      {
        const int px = tid >> 3, c8 = (tid & 7) * 8;
        const int ws = w0 + px + dx;
        __nv_bfloat16 v[8];
        if (w0 + px < W && hs >= 0 && hs < H && ws >= 0 && ws < W && ci0 + c8 < Cin) {
          const uint4 u = *reinterpret_cast<const uint4*>(X + (((size_t)n * H + hs) * W + ws) * xstride + xcoff + ci0 + c8);
          *reinterpret_cast<uint4*>(v) = u;
        } else {
#pragma unroll
          for (int e = 0; e < 8; ++e) v[e] = __float2bfloat16_rn(0.f);
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) Bs[c8 + e][px] = v[e];
      }
      __syncthreads();
      if (dbias && t == 4 && ci0 == 0 && tid < 64) {
        for (int px = 0; px < 16; ++px) bsum += __bfloat162float(As[tid][px]);
      }
      uint32_t a[4];
      const int r0 = warp * 16 + g;
      a[0] = ld_smem_u32(&As[r0][2 * tq]);
      a[1] = ld_smem_u32(&As[r0 + 8][2 * tq]);
      a[2] = ld_smem_u32(&As[r0][2 * tq + 8]);
      a[3] = ld_smem_u32(&As[r0 + 8][2 * tq + 8]);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        uint32_t b[2];
        b[0] = ld_smem_u32(&Bs[j * 8 + g][2 * tq]);
        b[1] = ld_smem_u32(&Bs[j * 8 + g][2 * tq + 8]);
        mma_bf16(acc[j], a, b);
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int co = co0 + warp * 16 + g + 8 * half;
      if (co >= Cout) continue;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int ci = ci0 + j * 8 + 2 * tq + e;
        if (ci >= Cin) continue;
        atomicAdd(&dW[((size_t)t * Cout + co) * Cin + ci], acc[j][2 * half + e]);
      }
    }
  }
  if (dbias && t == 4 && ci0 == 0 && tid < 64 && co0 + tid < Cout) atomicAdd(&dbias[co0 + tid], bsum);
}

// fp32 master weights (forward layout [t][co][ci]) -> bf16 forward layout and
// the bf16 data-gradient layout Wd[8 - t][ci][co].
__global__ void nn_weights_kernel(const float* __restrict__ Wm, int Cin, int Cout, __nv_bfloat16* __restrict__ Wf,
                                  __nv_bfloat16* __restrict__ Wd) {
  const int total = 9 * Cout * Cin;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int t = i / (Cout * Cin), rem = i % (Cout * Cin), co = rem / Cin, ci = rem % Cin;
    const __nv_bfloat16 v = __float2bfloat16_rn(Wm[i]);
    Wf[i] = v;
    if (Wd) Wd[((size_t)(8 - t) * Cin + ci) * Cout + co] = v;
  }
}

// dY *= (Y > 0) over channels [coff, coff + C) of a stride-channel buffer
// (Y is the ReLU output of the layer).
__global__ void nn_relu_bwd_kernel(__nv_bfloat16* __restrict__ dY, const __nv_bfloat16* __restrict__ Y, int64_t npix,
                                   int C, int dstride, int dcoff, int ystride, int ycoff) {
  const int64_t total = npix * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / C;
    const int c = (int)(i % C);
    if (!(__bfloat162float(Y[p * ystride + ycoff + c]) > 0.f)) dY[p * dstride + dcoff + c] = __float2bfloat16_rn(0.f);
  }
}

// 2 x 2 average pool (H, W even): Y[n, h, w, c] = mean of the 4 inputs.
__global__ void nn_pool2_kernel(const __nv_bfloat16* __restrict__ X, int N, int H, int W, int C, int xstride, int xcoff,
                                __nv_bfloat16* __restrict__ Y, int ystride, int ycoff) {
  const int Ho = H / 2, Wo = W / 2;
  const int64_t total = (int64_t)N * Ho * Wo * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t q = i / C;
    const int wo = (int)(q % Wo), ho = (int)((q / Wo) % Ho), n = (int)(q / ((int64_t)Wo * Ho));
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      s += __bfloat162float(X[(((size_t)n * H + 2 * ho + (k >> 1)) * W + 2 * wo + (k & 1)) * xstride + xcoff + c]);
    Y[(((size_t)n * Ho + ho) * Wo + wo) * ystride + ycoff + c] = __float2bfloat16_rn(0.25f * s);
  }
}

// dX (+)= dY / 4 spread over each 2 x 2 block.  accumulate: add to dX.
__global__ void nn_pool2_bwd_kernel(const __nv_bfloat16* __restrict__ dY, int N, int H, int W, int C, int dstride,
                                    int dcoff, __nv_bfloat16* __restrict__ dX, int xstride, int xcoff, int accumulate) {
  const int Ho = H / 2, Wo = W / 2;
  const int64_t total = (int64_t)N * H * W * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t q = i / C;
    const int w = (int)(q % W), h = (int)((q / W) % H), n = (int)(q / ((int64_t)W * H));
    const float g = 0.25f * __bfloat162float(dY[(((size_t)n * Ho + h / 2) * Wo + w / 2) * dstride + dcoff + c]);
    __nv_bfloat16& o = dX[q * xstride + xcoff + c];
    o = __float2bfloat16_rn(accumulate ? __bfloat162float(o) + g : g);
  }
}

// nearest 2x upsampling into channels [ycoff, ycoff + C) of Y (2H x 2W).
__global__ void nn_up2_kernel(const __nv_bfloat16* __restrict__ X, int N, int H, int W, int C, int xstride, int xcoff,
                              __nv_bfloat16* __restrict__ Y, int ystride, int ycoff) {
  const int Ho = 2 * H, Wo = 2 * W;
  const int64_t total = (int64_t)N * Ho * Wo * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t q = i / C;
    const int wo = (int)(q % Wo), ho = (int)((q / Wo) % Ho), n = (int)(q / ((int64_t)Wo * Ho));
    Y[q * ystride + ycoff + c] = X[(((size_t)n * H + ho / 2) * W + wo / 2) * xstride + xcoff + c];
  }
}

// dX = sum of dY over each 2 x 2 block (dY: 2H x 2W).
__global__ void nn_up2_bwd_kernel(const __nv_bfloat16* __restrict__ dY, int N, int H, int W, int C, int dstride,
                                  int dcoff, __nv_bfloat16* __restrict__ dX, int xstride, int xcoff) {
  const int64_t total = (int64_t)N * H * W * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t q = i / C;
    const int w = (int)(q % W), h = (int)((q / W) % H), n = (int)(q / ((int64_t)W * H));
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      s += __bfloat162float(dY[(((size_t)n * 2 * H + 2 * h + (k >> 1)) * 2 * W + 2 * w + (k & 1)) * dstride + dcoff + c]);
    dX[q * xstride + xcoff + c] = __float2bfloat16_rn(s);
  }
}

// Squared error over the central box [m, H - m) x [m, W - m) and the first
// `nc` of C channels: loss (+)= sum (pred - target)^2 / count; dpred (bf16)
// = 2 (pred - target) / count there, 0 elsewhere.
__global__ void nn_mse_kernel(const float* __restrict__ pred, const float* __restrict__ target, int N, int H, int W,
                              int C, int nc, int m, float inv_count, __nv_bfloat16* __restrict__ dpred,
                              float* __restrict__ loss) {
  const int64_t total = (int64_t)N * H * W * C;
  float local = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t q = i / C;
    const int w = (int)(q % W), h = (int)((q / W) % H);
    float gr = 0.f;
    if (c < nc && h >= m && h < H - m && w >= m && w < W - m) {
      const float d = pred[i] - target[i];
      local += d * d;
      gr = 2.f * d * inv_count;
    }
    if (dpred) dpred[i] = __float2bfloat16_rn(gr);
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, local * inv_count);
}

// Adam on float32 parameters (Kingma & Ba 2015), bias-corrected step t.
__global__ void nn_adam_kernel(float* __restrict__ p, const float* __restrict__ grad, float* __restrict__ m,
                               float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                               float c2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gr = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * gr;
    const float vi = b2 * v[i] + (1.f - b2) * gr * gr;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// Network input from the march rasters of a window (NHWC bf16, 16
// channels: heights above the window's ground of the building DSM, the
// canopy top and the trunk zone, each / 40 m; the rest 0).  origin (r0, c0)
// of each of the n windows in the site grid; cells outside the grid read 0.
__global__ void nn_input_kernel(const float* __restrict__ dsm, const float* __restrict__ vegdsm,
                                const float* __restrict__ vegdsm2, const float* __restrict__ dem, int rows, int cols,
                                const int2* __restrict__ origins, int n, int S, __nv_bfloat16* __restrict__ X) {
  const int64_t total = (int64_t)n * S * S;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int w = (int)(i % S), h = (int)((i / S) % S), k = (int)(i / ((int64_t)S * S));
    const int r = origins[k].x + h, c = origins[k].y + w;
    float f0 = 0.f, f1 = 0.f, f2 = 0.f;
    if (r >= 0 && r < rows && c >= 0 && c < cols) {
      const size_t p = (size_t)r * cols + c;
      const float g = dem ? dem[p] : 0.f;
      f0 = (dsm[p] - g) * (1.f / 40.f);
      f1 = vegdsm[p] > 0.f ? (vegdsm[p] - g) * (1.f / 40.f) : 0.f;
      f2 = vegdsm2[p] > 0.f ? (vegdsm2[p] - g) * (1.f / 40.f) : 0.f;
    }
    __nv_bfloat16* o = X + i * 16;
    o[0] = __float2bfloat16_rn(f0);
    o[1] = __float2bfloat16_rn(f1);
    o[2] = __float2bfloat16_rn(f2);
#pragma unroll
    for (int c2 = 3; c2 < 16; ++c2) o[c2] = __float2bfloat16_rn(0.f);
  }
}

}  // namespace sw100
