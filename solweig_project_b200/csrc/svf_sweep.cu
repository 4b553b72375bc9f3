// SVF patch sweep: all 153 sky patches of one site in one launch.
//
// Reference: solweig_gpu/shadow.py:166-322 (shadow(), one patch march) and
// shadow.py:409-625 (svf_calculator: patch loop, annulus weights, tails).
//
// One thread owns one pixel and marches every patch for it; the per-patch
// step tables (dx, dy, dz), built on the host with the reference's float32
// trigonometry, are read as warp-uniform broadcasts.  Each step gathers one
// float4 {dsm, vegdsm, vegdsm2, bush} at the shifted source: all lanes of a
// warp shift by the same (dx, dy), so the gather is a contiguous 512-byte
// row segment served from L1/L2 (consecutive steps shift by at most one
// pixel).  The 15 SVF accumulators are updated in the reference's order
// (patch-major, annulus-minor), so the sums are bit-identical; the three
// patch masks are packed into 5-word bit cubes per pixel (60 B/px instead of
// the reference's 1836 B/px of float cubes).
#include <climits>
#include <cmath>

#include "sw_common.cuh"

namespace sw100 {

struct SvfAcc {
  float svf, svfE, svfS, svfW, svfN;
  float veg, vegE, vegS, vegW, vegN;
  float aveg, avegE, avegS, avegW, avegN;
};

// One patch march for one pixel (shadow.py:228-316).  Returns final sh
// (1 = sky visible), vegsh and vbshvegsh as floats.  COUNT: add the number
// of source gathers the march executes to *ns (the counting instantiation
// of the sweep; the plain one compiles the counter away).
template <bool COUNT = false>
__device__ __forceinline__ void march_patch(const float4* __restrict__ src4, int rows, int cols, int r,
                                            int c, float a, float veg2_p, float bush_p,
                                            const sw100_step* __restrict__ steps, int n,
                                            const uint32_t* __restrict__ bflags, bool bush_any,
                                            float vmax, float& sh_out, float& veg_out, float& vb_out,
                                            int* ns = nullptr) {
  const bool bushplant = bush_p > 1.f;
  float f = a;
  float sh = 0.f;
  float vegsh = bushplant ? 1.f : 0.f;  // zeros + bushplant
  int vbsh = 0;                         // integer count of vegsh over steps >= 2
  float g = 0.f;
  const bool may_exit = !(bush_any && bushplant);
  for (int k = 0; k < n; ++k) {
    const sw100_step st = load_step(&steps[k]);
    const int sr = r + st.dx, sc = c + st.dy;
    const float dz = st.dz;
    float temp = 0.f, tv = 0.f, tv2 = 0.f, tb = 0.f;
    const bool inb = in_grid(sr, sc, rows, cols);
    if (inb) {
      if (COUNT) ++*ns;
      const float4 v = __ldg(&src4[(size_t)sr * cols + sc]);
      temp = __fsub_rn(v.x, dz);
      tv = __fsub_rn(v.y, dz);
      tv2 = __fsub_rn(v.z, dz);
      tb = __fsub_rn(v.w, dz);
    }
    f = tmax(f, temp);
    if (f > a) sh = 1.f;
    else if (f <= a) sh = 0.f;
    const bool fab = tv > a;
    const bool gab = tv2 > a;
    const float vegsh2 = (fab ? 1.f : 0.f) - (gab ? 1.f : 0.f);
    vegsh = tmax(vegsh, vegsh2);
    if (vegsh * sh > 0.f) vegsh = 0.f;
    vbsh += (vegsh > 0.f) ? 1 : 0;
    if (k == 0) {
      float first = __fsub_rn(tv, temp);
      if (first <= 0.f) first = 1000.f;
      if (first < dz) vegsh = 1.f;
      vegsh = vegsh * ((veg2_p > a) ? 1.f : 0.f);
      vbsh = 0;
    }
    if (bush_any && bflags[k]) {
      g = tmax(g, tb);
      g = g * (bushplant ? 1.f : 0.f);
    }
    if (may_exit && k >= 1) {
      // nothing later can change sh / vegsh / vbsh>0: building shadow is
      // final, or no source can rise above this pixel any more -- the ray
      // has left the grid (shifts grow monotonically, so it stays out and
      // reads zeros) or even the highest source minus the growing drop stays
      // at or below the pixel.  Both need a >= 0 (zeros never exceed it).
      const bool done = (sh == 1.f) || (a >= 0.f && (!inb || __fsub_rn(vmax, dz) <= a));
      if (done) {
        if (vegsh > 0.f && vbsh == 0 && k + 1 < n) vbsh = 1;
        break;
      }
    }
  }
  sh = 1.f - sh;
  float vb = (vbsh > 0) ? 1.f : 0.f;
  vb = vb - vegsh;
  if (bush_any) {
    g = g - bush_p;
    if (g > 0.f) g = 1.f;
    if (g < 0.f) g = 0.f;
    vegsh = vegsh - (bushplant ? 1.f : 0.f) + g;
    if (vegsh < 0.f) vegsh = 0.f;
  }
  if (vegsh > 0.f) vegsh = 1.f;
  vegsh = 1.f - vegsh;
  vb = 1.f - vb;
  sh_out = sh;
  veg_out = vegsh;
  vb_out = vb;
}

// The same march for a pixel that grows no bush shadow, on finite inputs.
// There the running maximum f only matters through "f > a", which turns on
// at the first source with height - dz > a and stays on; building shadow
// then zeroes the vegetation state for good, so the march ends there.
// vegsh and the "vbshvegsh ever counted" flag are booleans.  Returns final
// (sh, vegsh, vbshvegsh) with values as march_patch.
// Steps flagged SW100_STEP_SKIP8 whose 8-step source bound minus the step's
// drop is at or below the pixel cannot shade it or add vegetation: they are
// passed over 8 at a time (SkipMap, sw_common.cuh).
// CHECKED false: the caller has shown that every step of the march stays in
// the grid (the last step's cell is in it; the shifts grow monotonically).
template <bool CHECKED = true, bool COUNT = false>
__device__ __forceinline__ void march_patch_fast(const float4* __restrict__ src4, int rows, int cols, int r, int c,
                                                 float a, float veg2_p, const sw100_step* __restrict__ steps, int n,
                                                 float vmax, float& sh_out, float& veg_out, float& vb_out,
                                                 SkipMap skip = SkipMap{nullptr, 0}, int* ns = nullptr) {
  bool sh = false, vegsh = false, vb_any = false;
  if (n > 0) {
    // first step (index 1 of shadow.py): the trunk-zone rule of :288-293
    const sw100_step st = load_step(&steps[0]);
    const int sr = r + st.dx, sc = c + st.dy;
    float temp = 0.f, tv = 0.f, tv2 = 0.f;
    if (!CHECKED || in_grid(sr, sc, rows, cols)) {
      if (COUNT) ++*ns;
      const float4 v = __ldg(&src4[(size_t)sr * cols + sc]);
      temp = __fsub_rn(v.x, st.dz);
      tv = __fsub_rn(v.y, st.dz);
      tv2 = __fsub_rn(v.z, st.dz);
    }
    sh = temp > a;
    vegsh = (tv > a) && !(tv2 > a) && !sh;
    float first = __fsub_rn(tv, temp);
    if (first <= 0.f) first = 1000.f;
    if (first < st.dz) vegsh = true;
    vegsh = vegsh && (veg2_p > a);
    if (sh) {
      if (n > 1) vegsh = false;  // the next step zeroes it under building shadow
    } else {
      const bool can_skip = skip.m != nullptr && a >= 0.f;
      for (int k = 1; k < n; ++k) {
        const sw100_step sk = load_step(&steps[k]);
        const int rr = r + sk.dx, cc = c + sk.dy;
        if (CHECKED && !in_grid(rr, cc, rows, cols)) {
          // zeros from here on: shadow only for a pixel below 0
          if (0.f > a) { sh = true; vegsh = false; }
          else vb_any = vb_any || vegsh;
          break;
        }
        if (can_skip && (sk.flags & SW100_STEP_SKIP8) && sk.dz >= 0.f &&
            __fsub_rn(skip_bound(skip, rr, cc), sk.dz) <= a) {
          vb_any = vb_any || vegsh;  // all each of the 8 skipped steps would do
          k += 7;
          continue;
        }
        if (COUNT) ++*ns;
        const float4 v = __ldg(&src4[(size_t)rr * cols + cc]);
        if (__fsub_rn(v.x, sk.dz) > a) { sh = true; vegsh = false; break; }
        vegsh = vegsh || ((__fsub_rn(v.y, sk.dz) > a) && !(__fsub_rn(v.z, sk.dz) > a));
        vb_any = vb_any || vegsh;
        if (a >= 0.f && __fsub_rn(vmax, sk.dz) <= a) break;
      }
    }
  }
  const float vegf = vegsh ? 1.f : 0.f;
  sh_out = sh ? 0.f : 1.f;
  veg_out = 1.f - vegf;
  vb_out = 1.f - ((vb_any ? 1.f : 0.f) - vegf);
}

// Adds patch q's (sh, vegsh, vbshvegsh) to the 15 SVF sums in the
// reference's order: annulus by annulus, each direction sum after the
// isotropic one (shadow.py:560-585).
__device__ __forceinline__ void svf_add_patch(SvfAcc& A, const sw100_svf_plan& plan, int q, float sh, float veg,
                                              float vb) {
  const int ring = plan.ring[q];
  const int fl = plan.dir_flags[q];
  const int na = plan.ring_annuli[ring];
  for (int k = 0; k < na; ++k) {
    const float wi = plan.w_iso[ring][k];
    const float wa = plan.w_aniso[ring][k];
    A.svf = A.svf + wi * sh;
    const float wsh_ = wa * sh;
    if (fl & 1) A.svfE = A.svfE + wsh_;
    if (fl & 2) A.svfS = A.svfS + wsh_;
    if (fl & 4) A.svfW = A.svfW + wsh_;
    if (fl & 8) A.svfN = A.svfN + wsh_;
    A.veg = A.veg + wi * veg;
    A.aveg = A.aveg + wi * vb;
    const float wv = wa * veg, wb = wa * vb;
    if (fl & 1) { A.vegE = A.vegE + wv; A.avegE = A.avegE + wb; }
    if (fl & 2) { A.vegS = A.vegS + wv; A.avegS = A.avegS + wb; }
    if (fl & 4) { A.vegW = A.vegW + wv; A.avegW = A.avegW + wb; }
    if (fl & 8) { A.vegN = A.vegN + wv; A.avegN = A.avegN + wb; }
  }
}

// Patch bits of one march result.  Marches of at most one step leave
// vbshvegsh in {1, 2}: their bit keeps "== 1"; every other patch keeps
// "!= 0" (values {0, 1}).
__device__ __forceinline__ void svf_set_bits(uint32_t* wsh, uint32_t* wveg, uint32_t* wvb, int q, int n, float sh,
                                             float veg, float vb) {
  const uint32_t bit = 1u << (q & 31);
  if (sh != 0.f) wsh[q >> 5] |= bit;
  if (veg != 0.f) wveg[q >> 5] |= bit;
  if (n <= 1 ? (vb == 1.f) : (vb != 0.f)) wvb[q >> 5] |= bit;
}

// Time-loop statics of a pixel from its svf and svfveg
// (utci_process.py:864-897): svfbuveg, tan(asvf) with asvf =
// acos(sqrt(svf)) and tan(svfalfa) with svfalfa = asin(exp(log(1 - tmp) /
// 2)), tmp = max(svf + svfveg - 1, 0); every float32 operation of the
// reference rounded once, transcendentals evaluated in double.
__device__ __forceinline__ void svf_statics(float svf, float veg, float trans_veg, float& buveg, float& hsvf,
                                            float& tan_alfa) {
  buveg = svf - (1.f - veg) * (1.f - trans_veg);
  const float s = (float)sqrt((double)svf);
  const float asvf = (float)acos((double)s);
  hsvf = (float)tan((double)asvf);
  float tmp = svf + veg - 1.f;
  if (tmp < 0.f) tmp = 0.f;
  const float lg = (float)log((double)(1.f - tmp));
  const float ex = (float)exp((double)(lg / 2.f));
  const float alfa = (float)asin((double)ex);
  tan_alfa = (float)tan((double)alfa);
}

// The three statics planes of an SVF result given as planes (a bundle that
// did not come from this library's sweep): planes 16-18 from planes 0 and 11.
__global__ void svf_statics_kernel(float* __restrict__ planes, int64_t npix, float trans_veg) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (int64_t)gridDim.x * blockDim.x) {
    float b, h, t;
    svf_statics(planes[p], planes[11 * npix + p], trans_veg, b, h, t);
    planes[16 * npix + p] = b;
    planes[17 * npix + p] = h;
    planes[18 * npix + p] = t;
  }
}

// Tails, clamps (shadow.py:587-613), the 16 SVF planes, the three
// time-loop statics and the bit cubes of pixel p.
__device__ __forceinline__ void svf_finish(SvfAcc& A, const sw100_svf_plan& plan, float veg2_p, size_t p,
                                           size_t npix, const uint32_t* wsh, const uint32_t* wveg,
                                           const uint32_t* wvb, float* __restrict__ out,
                                           uint32_t* __restrict__ bits) {
  const float tail = plan.tail;
  A.svfS = A.svfS + tail;
  A.svfW = A.svfW + tail;
  auto clamp1 = [](float& x) { if (x > 1.f) x = 1.f; };
  clamp1(A.svf); clamp1(A.svfE); clamp1(A.svfS); clamp1(A.svfW); clamp1(A.svfN);
  const float last = (veg2_p == 0.f) ? tail : 0.f;
  A.vegS = A.vegS + last;
  A.vegW = A.vegW + last;
  A.avegS = A.avegS + last;
  A.avegW = A.avegW + last;
  clamp1(A.veg); clamp1(A.vegE); clamp1(A.vegS); clamp1(A.vegW); clamp1(A.vegN);
  clamp1(A.aveg); clamp1(A.avegE); clamp1(A.avegS); clamp1(A.avegW); clamp1(A.avegN);
  const float total = A.svf - (1.f - A.veg) * (1.f - plan.trans);
  // reference tuple order (shadow.py:625) without the cubes, then SVFtotal
  const float vals[16] = {A.svf,  A.aveg,  A.svfE, A.avegE, A.vegE, A.svfN, A.avegN, A.vegN,
                          A.svfS, A.avegS, A.vegS, A.veg,   A.svfW, A.avegW, A.vegW, total};
#pragma unroll
  for (int k = 0; k < 16; ++k) out[k * npix + p] = vals[k];
  svf_statics(A.svf, A.veg, plan.trans_veg, out[16 * npix + p], out[17 * npix + p], out[18 * npix + p]);
#pragma unroll
  for (int w = 0; w < SW100_CUBE_WORDS; ++w) {
    bits[(0 * SW100_CUBE_WORDS + w) * npix + p] = wsh[w];
    bits[(1 * SW100_CUBE_WORDS + w) * npix + p] = wveg[w];
    bits[(2 * SW100_CUBE_WORDS + w) * npix + p] = wvb[w];
  }
}

// A patch's steps clamped into the step table of n_steps entries (a plan
// built by the host library is always inside; a malformed plan from another
// caller then reads no memory outside the table).
__device__ __forceinline__ void clamp_patch(int off, int cnt, int n_steps, int& o, int& n) {
  o = min(max(off, 0), n_steps);
  n = min(max(cnt, 0), n_steps - o);
}

// Copies the plan into shared memory and clamps every index it holds
// (patch count, ring and annulus counts, step ranges) to the arrays they
// index.  Every thread of the block calls it; it ends with a barrier.
__device__ __forceinline__ void load_plan(const sw100_svf_plan* __restrict__ plan_g, sw100_svf_plan& plan,
                                          int n_steps) {
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
  const int* s = reinterpret_cast<const int*>(plan_g);
  int* d = reinterpret_cast<int*>(&plan);
  const int nw = sizeof(sw100_svf_plan) / 4;
  for (int i = tid; i < nw; i += nthr) d[i] = s[i];
  __syncthreads();
  if (tid == 0) plan.n_patches = min(max(plan.n_patches, 0), SW100_MAX_PATCHES);
  for (int q = tid; q < SW100_MAX_PATCHES; q += nthr) {
    int o, n;
    clamp_patch(plan.step_offset[q], plan.step_count[q], n_steps, o, n);
    plan.step_offset[q] = o;
    plan.step_count[q] = n;
    plan.ring[q] = min(max(plan.ring[q], 0), SW100_MAX_RINGS - 1);
  }
  for (int r = tid; r < SW100_MAX_RINGS; r += nthr) plan.ring_annuli[r] = min(max(plan.ring_annuli[r], 0), SW100_MAX_ANNULI);
  __syncthreads();
}

// The 153 patch marches, the sums and the outputs of pixel (r, c).
// COUNT: also add the source gathers executed to *ns.
template <bool COUNT = false>
__device__ __forceinline__ void svf_sweep_pixel(const float4* __restrict__ src4, int rows, int cols,
                                                const sw100_svf_plan& plan, const sw100_step* __restrict__ steps,
                                                const uint32_t* __restrict__ bflags, float vmax,
                                                float* __restrict__ out, uint32_t* __restrict__ bits, int r, int c,
                                                SkipMap skip = SkipMap{nullptr, 0}, int* ns = nullptr) {
  const size_t npix = (size_t)rows * cols;
  const size_t p = (size_t)r * cols + c;
  const float4 self = src4[p];
  const float a = self.x, veg2_p = self.z, bush_p = self.w;
  const bool bush_any = plan.bush_any != 0;
  const bool fast = plan.all_finite != 0 && !(bush_any && bush_p > 1.f);

  SvfAcc A = {};
  uint32_t wsh[SW100_CUBE_WORDS] = {0, 0, 0, 0, 0};
  uint32_t wveg[SW100_CUBE_WORDS] = {0, 0, 0, 0, 0};
  uint32_t wvb[SW100_CUBE_WORDS] = {0, 0, 0, 0, 0};

  for (int q = 0; q < plan.n_patches; ++q) {
    const int off = plan.step_offset[q];
    const int n = plan.step_count[q];
    float sh, veg, vb;
    if (fast)
      {
        // a march whose last cell is in the grid never leaves it
        bool inside = false;
        if (n > 0) {
          const sw100_step last = load_step(&steps[off + n - 1]);
          inside = in_grid(r + last.dx, c + last.dy, rows, cols);
        }
        if (inside)
          march_patch_fast<false, COUNT>(src4, rows, cols, r, c, a, veg2_p, steps + off, n, vmax, sh, veg, vb, skip,
                                         ns);
        else
          march_patch_fast<true, COUNT>(src4, rows, cols, r, c, a, veg2_p, steps + off, n, vmax, sh, veg, vb, skip,
                                        ns);
      }
    else
      march_patch<COUNT>(src4, rows, cols, r, c, a, veg2_p, bush_p, steps + off, n,
                         bush_any ? bflags + off : nullptr, bush_any, vmax, sh, veg, vb, ns);
    svf_set_bits(wsh, wveg, wvb, q, n, sh, veg, vb);
    svf_add_patch(A, plan, q, sh, veg, vb);
  }
  svf_finish(A, plan, veg2_p, p, npix, wsh, wveg, wvb, out, bits);
}

// The skip map of a site: for each 8 x 8 block, the largest source height
// (dsm, vegdsm, vegdsm2) over the block and its neighbours; NaN propagates
// (a NaN bound never passes the skip test; the sign of a zero maximum does
// not matter to the test).  One warp per block: the lanes stride over the
// (up to) 24 x 24 cells and reduce with shuffles.
__device__ __forceinline__ void skipmap_block_warp(const float4* __restrict__ src4, int rows, int cols,
                                                   float* __restrict__ m, int ccol, int b, int lane) {
  const int br = b / ccol, bc = b % ccol;
  const int r0 = max(0, (br - 1) * 8), r1 = min(rows, (br + 2) * 8);
  const int c0 = max(0, (bc - 1) * 8), c1 = min(cols, (bc + 2) * 8);
  const int w = c1 - c0, n = (r1 - r0) * w;
  float v = -INFINITY;
  for (int i = lane; i < n; i += 32) {
    const float4 s = src4[(size_t)(r0 + i / w) * cols + (c0 + i % w)];
    v = tmax(v, tmax(s.x, tmax(s.y, s.z)));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = tmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  if (lane == 0) m[b] = v;
}

__global__ void svf_skipmap_kernel(const float4* __restrict__ src4, int rows, int cols, float* __restrict__ m,
                                   int crow, int ccol) {
  const int b = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (b >= crow * ccol) return;  // whole warps: the block count is a multiple of 32 threads
  skipmap_block_warp(src4, rows, cols, m, ccol, b, threadIdx.x & 31);
}

// Persistent sweep: as many 128-thread blocks as fit on the device at once;
// each warp takes the next 8 x 4 pixel patch (k: rows 4 (k / pc) .. + 3,
// columns 8 (k % pc) .. + 7, pc = ceil(cols / 8)) from the counter *next
// (zero at launch) until all n_patch are taken.  The patches go out in grid
// order, so the warps at work march neighbouring pixels; a warp that drew
// short marches takes the next patch at once instead of idling until its
// block is done, and there is no last partial wave of blocks.
__global__ void __launch_bounds__(128, 12) svf_sweep_kernel(
    const float4* __restrict__ src4, int rows, int cols, const sw100_svf_plan* __restrict__ plan_g,
    const sw100_step* __restrict__ steps, const uint32_t* __restrict__ bflags, float vmax,
    float* __restrict__ out, uint32_t* __restrict__ bits, int n_steps, const float* __restrict__ skipmap,
    unsigned int* __restrict__ next, int n_patch) {
  __shared__ sw100_svf_plan plan;
  load_plan(plan_g, plan, n_steps);
  const int lane = threadIdx.x & 31, pcols = (cols + 7) >> 3;
  for (;;) {
    int k = 0;
    if (lane == 0) k = (int)atomicAdd(next, 1u);
    k = __shfl_sync(0xffffffffu, k, 0);
    if (k >= n_patch) break;  // warp-uniform
    const int r = (k / pcols) * 4 + (lane >> 3), c = (k % pcols) * 8 + (lane & 7);
    if (r < rows && c < cols)
      svf_sweep_pixel(src4, rows, cols, plan, steps, bflags, vmax, out, bits, r, c, SkipMap{skipmap, pcols});
  }
}

// The same sweep, also counting the source gathers its marches execute
// (each gathers the 12 bytes dsm / vegdsm / vegdsm2 the survey's step
// counts are defined on): the algorithmic bytes of a launch are 12 x this
// count.  Results are identical to svf_sweep_kernel's; the count is
// reduced per warp and added to *executed with one atomic per warp.
__global__ void __launch_bounds__(128, 12) svf_sweep_count_kernel(
    const float4* __restrict__ src4, int rows, int cols, const sw100_svf_plan* __restrict__ plan_g,
    const sw100_step* __restrict__ steps, const uint32_t* __restrict__ bflags, float vmax,
    float* __restrict__ out, uint32_t* __restrict__ bits, int n_steps, const float* __restrict__ skipmap,
    unsigned long long* __restrict__ executed) {
  __shared__ sw100_svf_plan plan;
  load_plan(plan_g, plan, n_steps);
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  int ns = 0;
  if (r < rows && c < cols)
    svf_sweep_pixel<true>(src4, rows, cols, plan, steps, bflags, vmax, out, bits, r, c,
                          SkipMap{skipmap, (cols + 7) / 8}, &ns);
  unsigned long long v = (unsigned long long)ns;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if ((threadIdx.x + threadIdx.y * blockDim.x) % 32 == 0) atomicAdd(executed, v);
}

// ------------------------------------------------------------- batches
// Tile t of a batch: pixel (r, c) of this thread, and whether it exists.
__device__ __forceinline__ bool batch_pixel(const sw100_batch_site& S, const sw100_tile& T, int& r, int& c) {
  c = T.tx * blockDim.x + threadIdx.x;
  r = T.ty * blockDim.y + threadIdx.y;
  return r < S.rows && c < S.cols;
}

// SVF sweep of every site of a batch, tiles taken in list order.
__global__ void __launch_bounds__(128, 10) svf_sweep_batch_kernel(const sw100_batch_site* __restrict__ sites,
                                                              const sw100_tile* __restrict__ tiles, int n_tiles) {
  __shared__ sw100_svf_plan plan;
  for (int i = blockIdx.x; i < n_tiles; i += gridDim.x) {
    const sw100_tile T = tiles[i];
    const sw100_batch_site& S = sites[T.site];
    __syncthreads();  // the previous tile is done with the shared plan
    load_plan(S.plan, plan, S.svf_steps);
    int r, c;
    if (batch_pixel(S, T, r, c))
      svf_sweep_pixel(reinterpret_cast<const float4*>(S.src4), S.rows, S.cols, plan, S.steps,
                      S.site.bush_any ? S.bflags : nullptr, S.site.vmax, S.svf_planes, S.svf_bits, r, c,
                      SkipMap{S.skipmap, (S.cols + 7) / 8});
  }
}

// Skip maps of the sites of a batch: grid.y = site, blocks stride over the
// site's 8 x 8 cell blocks.
__global__ void __launch_bounds__(128) skipmap_batch_kernel(const sw100_batch_site* __restrict__ sites) {
  const sw100_batch_site& S = sites[blockIdx.y];
  if (S.skipmap == nullptr) return;
  const int ccol = (S.cols + 7) / 8, nb = ((S.rows + 7) / 8) * ccol;
  const int warps = (int)(gridDim.x * blockDim.x) >> 5;
  for (int b = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); b < nb; b += warps)
    skipmap_block_warp(reinterpret_cast<const float4*>(S.src4), S.rows, S.cols, S.skipmap, ccol, b,
                       threadIdx.x & 31);
}

// Packs {dsm, vegdsm, vegdsm2, bush} of every site of a batch.
__global__ void __launch_bounds__(128) pack_batch_kernel(const sw100_batch_site* __restrict__ sites,
                                                         const sw100_tile* __restrict__ tiles, int n_tiles) {
  for (int i = blockIdx.x; i < n_tiles; i += gridDim.x) {
    const sw100_tile T = tiles[i];
    const sw100_batch_site& S = sites[T.site];
    int r, c;
    if (!batch_pixel(S, T, r, c)) continue;
    const size_t p = (size_t)r * S.cols + c;
    reinterpret_cast<float4*>(S.src4)[p] =
        make_float4(S.site.dsm[p], S.site.vegdsm[p], S.site.vegdsm2[p], S.site.bush_any ? S.site.bush[p] : 0.f);
  }
}

// The whole-grid bush step flags of the sites of a batch that have bush
// (the tile list holds tiles of those sites only).
__global__ void __launch_bounds__(128) svf_bush_flags_batch_kernel(const sw100_batch_site* __restrict__ sites,
                                                                   const sw100_tile* __restrict__ tiles, int n_tiles) {
  for (int i = blockIdx.x; i < n_tiles; i += gridDim.x) {
    const sw100_tile T = tiles[i];
    const sw100_batch_site& S = sites[T.site];
    int r, c;
    if (!batch_pixel(S, T, r, c)) continue;
    const float4* src4 = reinterpret_cast<const float4*>(S.src4);
    const float4 self = src4[(size_t)r * S.cols + c];
    if (!(self.w > 0.f)) continue;
    const sw100_svf_plan* plan = S.plan;
    const int np = min(max(plan->n_patches, 0), SW100_MAX_PATCHES);
    for (int q = 0; q < np; ++q) {
      int off, n;
      clamp_patch(plan->step_offset[q], plan->step_count[q], S.svf_steps, off, n);
      for (int k = 0; k < n; ++k) {
        const sw100_step st = S.steps[off + k];
        const int sr = r + st.dx, sc = c + st.dy;
        float tv = 0.f;
        if (in_grid(sr, sc, S.rows, S.cols)) tv = __fsub_rn(src4[(size_t)sr * S.cols + sc].y, st.dz);
        if (tv > self.x && S.bflags[off + k] == 0u) atomicExch(&S.bflags[off + k], 1u);
      }
    }
  }
}

// Does the march of pixel (tr, tc) along this patch's steps read a cell of
// the edited rectangle [r0, r1] x [c0, c1], or is the pixel inside it?
// The patch's major shift is s * (k + 1) at step k along one axis and its
// minor shift moves by at most one cell per step, monotonically (checked on
// the host, which marks any other patch `SW100_CORRIDOR_ALWAYS`, and a
// patch whose result does not depend on the heights it reads
// `SW100_CORRIDOR_LOCAL`).  The steps
// whose major shift lands in the rectangle's band form one interval
// [ka, kb]; the minor shifts over it cover every integer between the
// interval's end values, so the test needs two step reads.
__device__ __forceinline__ bool svf_in_corridor(int tr, int tc, const sw100_step* __restrict__ st, int n,
                                                int desc, int r0, int r1, int c0, int c1) {
  if (tr >= r0 && tr <= r1 && tc >= c0 && tc <= c1) return true;
  const int axis = desc & 3;
  if (n <= 0 || axis == SW100_CORRIDOR_LOCAL) return false;
  if (axis == SW100_CORRIDOR_ALWAYS) return true;
  const bool neg = (desc & 4) != 0;
  const int tM = axis == 0 ? tr : tc, lo = axis == 0 ? r0 : c0, hi = axis == 0 ? r1 : c1;
  const int tm = axis == 0 ? tc : tr, mlo = axis == 0 ? c0 : r0, mhi = axis == 0 ? c1 : r1;
  int ka = neg ? tM - hi : lo - tM;  // range of k + 1
  int kb = neg ? tM - lo : hi - tM;
  ka = max(ka, 1);
  kb = min(kb, n);
  if (ka > kb) return false;
  const sw100_step sa = load_step(&st[ka - 1]), sb = load_step(&st[kb - 1]);
  const int ma = axis == 0 ? sa.dy : sa.dx, mb = axis == 0 ? sb.dy : sb.dx;
  return tm + max(ma, mb) >= mlo && tm + min(ma, mb) <= mhi;
}

// Windowed exact recompute after an edit of the march rasters inside the
// rectangle `rect` = (r0, r1, c0, c1), inclusive.  Pixels of `win` re-march
// only the patches whose march reads the rectangle (or that start in it),
// keep the stored bits of every other patch, and re-accumulate all sums in
// the sweep's order: the result equals a full sweep of the edited rasters
// bit for bit.  Pixels outside `win` are not touched (no march of theirs
// reaches the rectangle).  Bush rasters are excluded by the host (their
// whole-grid step flags would change).
__global__ void __launch_bounds__(128) svf_window_kernel(
    const float4* __restrict__ src4, int rows, int cols, const sw100_svf_plan* __restrict__ plan_g,
    const sw100_step* __restrict__ steps, const int32_t* __restrict__ corridor, float vmax, int4 rect, int4 win,
    float* __restrict__ out, uint32_t* __restrict__ bits, int n_steps) {
  __shared__ sw100_svf_plan plan;
  load_plan(plan_g, plan, n_steps);
  const int c = win.z + blockIdx.x * blockDim.x + threadIdx.x;
  const int r = win.x + blockIdx.y * blockDim.y + threadIdx.y;
  if (r > win.y || c > win.w) return;
  const size_t npix = (size_t)rows * cols;
  const size_t p = (size_t)r * cols + c;
  const float4 self = src4[p];
  const float a = self.x, veg2_p = self.z;
  const bool fast = plan.all_finite != 0;

  uint32_t osh[SW100_CUBE_WORDS], oveg[SW100_CUBE_WORDS], ovb[SW100_CUBE_WORDS];
#pragma unroll
  for (int w = 0; w < SW100_CUBE_WORDS; ++w) {
    osh[w] = bits[(0 * SW100_CUBE_WORDS + w) * npix + p];
    oveg[w] = bits[(1 * SW100_CUBE_WORDS + w) * npix + p];
    ovb[w] = bits[(2 * SW100_CUBE_WORDS + w) * npix + p];
  }
  SvfAcc A = {};
  uint32_t wsh[SW100_CUBE_WORDS] = {0, 0, 0, 0, 0};
  uint32_t wveg[SW100_CUBE_WORDS] = {0, 0, 0, 0, 0};
  uint32_t wvb[SW100_CUBE_WORDS] = {0, 0, 0, 0, 0};
  for (int q = 0; q < plan.n_patches; ++q) {
    const int off = plan.step_offset[q];
    const int n = plan.step_count[q];
    float sh, veg, vb;
    if (svf_in_corridor(r, c, steps + off, n, corridor[q], rect.x, rect.y, rect.z, rect.w)) {
      if (fast)
        march_patch_fast(src4, rows, cols, r, c, a, veg2_p, steps + off, n, vmax, sh, veg, vb);
      else
        march_patch(src4, rows, cols, r, c, a, veg2_p, 0.f, steps + off, n, nullptr, false, vmax, sh, veg, vb);
    } else {
      const uint32_t bit = 1u << (q & 31);
      const int w = q >> 5;
      sh = (osh[w] & bit) ? 1.f : 0.f;
      veg = (oveg[w] & bit) ? 1.f : 0.f;
      vb = (ovb[w] & bit) ? 1.f : (n <= 1 ? 2.f : 0.f);
    }
    svf_set_bits(wsh, wveg, wvb, q, n, sh, veg, vb);
    svf_add_patch(A, plan, q, sh, veg, vb);
  }
  svf_finish(A, plan, veg2_p, p, npix, wsh, wveg, wvb, out, bits);
}

__global__ void box_init_kernel(int* box) {
  if (threadIdx.x == 0) {
    box[0] = INT_MAX; box[1] = -1; box[2] = INT_MAX; box[3] = -1;
  }
}

// The patch marches of every (pixel, patch) pair of a box, one thread per
// pair, writing the pixels' patch bits (atomic bit updates: each thread
// owns its bit).  Followed by svf_window_kernel over the box with a
// rectangle that no march reads, which re-accumulates the planes from the
// new bits in the sweep's order.  Rasters without bush only.
__global__ void __launch_bounds__(128) svf_box_pairs_kernel(
    const float4* __restrict__ src4, int rows, int cols, const sw100_svf_plan* __restrict__ plan,
    const sw100_step* __restrict__ steps, float vmax, int4 box, uint32_t* __restrict__ bits, int n_steps) {
  const int bw = box.w - box.z + 1, bh = box.y - box.x + 1;
  const int np = min(max(plan->n_patches, 0), SW100_MAX_PATCHES);
  const int64_t total = (int64_t)bw * bh * np;
  const size_t npix = (size_t)rows * cols;
  const bool finite = plan->all_finite != 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(i % np);
    const int64_t px = i / np;
    const int r = box.x + (int)(px / bw), c = box.z + (int)(px % bw);
    const size_t p = (size_t)r * cols + c;
    const float4 self = src4[p];
    int off, n;
    clamp_patch(plan->step_offset[q], plan->step_count[q], n_steps, off, n);
    float sh, veg, vb;
    if (finite)
      march_patch_fast(src4, rows, cols, r, c, self.x, self.z, steps + off, n, vmax, sh, veg, vb);
    else
      march_patch(src4, rows, cols, r, c, self.x, self.z, 0.f, steps + off, n, nullptr, false, vmax, sh, veg, vb);
    const uint32_t bit = 1u << (q & 31);
    const int w = q >> 5;
    uint32_t* wsh = &bits[(0 * SW100_CUBE_WORDS + w) * npix + p];
    uint32_t* wveg = &bits[(1 * SW100_CUBE_WORDS + w) * npix + p];
    uint32_t* wvb = &bits[(2 * SW100_CUBE_WORDS + w) * npix + p];
    if (sh != 0.f) atomicOr(wsh, bit); else atomicAnd(wsh, ~bit);
    if (veg != 0.f) atomicOr(wveg, bit); else atomicAnd(wveg, ~bit);
    if (n <= 1 ? (vb == 1.f) : (vb != 0.f)) atomicOr(wvb, bit); else atomicAnd(wvb, ~bit);
  }
}

// Bounding box of the cells where two packed march sources differ (bit
// comparison of all four channels); box = {rmin, rmax, cmin, cmax}, set to
// {INT_MAX, -1, INT_MAX, -1} by the caller.
__global__ void diff_bbox_kernel(const float4* __restrict__ a, const float4* __restrict__ b, int rows, int cols,
                                 int* __restrict__ box) {
  const size_t n = (size_t)rows * cols;
  int rmin = INT_MAX, rmax = -1, cmin = INT_MAX, cmax = -1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int4 x = reinterpret_cast<const int4*>(a)[i];
    const int4 y = reinterpret_cast<const int4*>(b)[i];
    if (x.x != y.x || x.y != y.y || x.z != y.z || x.w != y.w) {
      const int r = (int)(i / cols), c = (int)(i % cols);
      rmin = min(rmin, r); rmax = max(rmax, r); cmin = min(cmin, c); cmax = max(cmax, c);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    rmin = min(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
    rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
    cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
    cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
  }
  if ((threadIdx.x & 31) == 0 && rmax >= 0) {
    atomicMin(&box[0], rmin); atomicMax(&box[1], rmax);
    atomicMin(&box[2], cmin); atomicMax(&box[3], cmax);
  }
}

// Whole-grid bush test of shadow.py:295 (`torch.max(fabovea * bush) > 0`):
// flag the steps at which any pixel with bush > 0 sees vegetation above it.
__global__ void svf_bush_flags_kernel(const float4* __restrict__ src4, int rows, int cols,
                                      const sw100_svf_plan* __restrict__ plan, const sw100_step* __restrict__ steps,
                                      uint32_t* __restrict__ flags, int n_steps) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  if (r >= rows || c >= cols) return;
  const float4 self = src4[(size_t)r * cols + c];
  if (!(self.w > 0.f)) return;
  const float a = self.x;
  const int np = min(max(plan->n_patches, 0), SW100_MAX_PATCHES);
  for (int q = 0; q < np; ++q) {
    int off, n;
    clamp_patch(plan->step_offset[q], plan->step_count[q], n_steps, off, n);
    for (int k = 0; k < n; ++k) {
      const sw100_step st = steps[off + k];
      const int sr = r + st.dx, sc = c + st.dy;
      float tv = 0.f;
      if (in_grid(sr, sc, rows, cols)) tv = __fsub_rn(src4[(size_t)sr * cols + sc].y, st.dz);
      if (tv > a && flags[off + k] == 0u) atomicExch(&flags[off + k], 1u);
    }
  }
}

// Dense (rows, cols, P) float cubes -> word-planar bit cubes.
__global__ void pack_cubes_kernel(const float* __restrict__ sh, const float* __restrict__ veg,
                                  const float* __restrict__ vb, size_t npix, int n_patches, Single5 single,
                                  uint32_t* __restrict__ bits) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npix; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t w0[SW100_CUBE_WORDS] = {}, w1[SW100_CUBE_WORDS] = {}, w2[SW100_CUBE_WORDS] = {};
    const float* a = sh + i * n_patches;
    const float* b = veg + i * n_patches;
    const float* c = vb + i * n_patches;
    for (int q = 0; q < n_patches; ++q) {
      const uint32_t bit = 1u << (q & 31);
      const bool one_step = single.w[q >> 5] & bit;
      if (a[q] != 0.f) w0[q >> 5] |= bit;
      if (b[q] != 0.f) w1[q >> 5] |= bit;
      if (one_step ? (c[q] == 1.f) : (c[q] != 0.f)) w2[q >> 5] |= bit;
    }
    for (int w = 0; w < SW100_CUBE_WORDS; ++w) {
      bits[(0 * SW100_CUBE_WORDS + w) * npix + i] = w0[w];
      bits[(1 * SW100_CUBE_WORDS + w) * npix + i] = w1[w];
      bits[(2 * SW100_CUBE_WORDS + w) * npix + i] = w2[w];
    }
  }
}

// Packs {dsm, vegdsm, vegdsm2, bush} into one float4 plane.
__global__ void pack4_kernel(const float* __restrict__ a, const float* __restrict__ b, const float* __restrict__ c,
                             const float* __restrict__ d, size_t n, float4* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = make_float4(a[i], b[i], c[i], d ? d[i] : 0.f);
}

}  // namespace sw100
