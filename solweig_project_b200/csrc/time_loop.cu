// The whole time loop of one site in one launch.
//
// Reference: solweig_gpu/utci_process.py:917-1067 (run_utci_window's loop)
// around solweig_gpu/solweig.py:1950-2311 (Solweig_2022a_calc) with
// cyl = 1, anisotropic_sky = 1, usevegdem = 1, onlyglobal = 1:
//   * ground view factors, 18 azimuths x `second` steps
//     (gvf_2018a / sunonsurface_2018a, solweig.py:75-402), including the
//     reference's stale-border temporaries (a ray that leaves the grid keeps
//     the last in-grid sample);
//   * thermal lag TsWaveDelay_2015a (solweig.py:451-488) with the six state
//     planes held in registers across the steps;
//   * cylindric_wedge, Kdown, Kup_veg_2015a, Kside_veg_v2022a
//     (solweig.py:404-449, 490-522, 564-832);
//   * Lcyl_v2022a / define_patch_characteristics (solweig.py:1439-1760);
//   * Tmrt (solweig.py:2291-2299) and UTCI (calculate_utci.py:259-330),
//     NaN outside buildings == 1 (utci_process.py:1047-1049).
//
// One thread owns one pixel for all steps.  Per-step scalars and the per-patch
// constant table are staged in shared memory once per step for the block.
// The 153-patch sums read the packed bit cubes of the SVF sweep (60 B per
// pixel) instead of three float cubes; their per-patch increments are host
// constants evaluated in the reference's association, so each sum is the
// same sequence of float32 additions (float64 where the reference promotes).
#include <cmath>
#include <cstddef>
#include <type_traits>

#include "sw_common.cuh"
#include "sw_internal.cuh"
#include "utci_series.cuh"

namespace sw100 {

constexpr int kMaxPatchSmem = 153;
constexpr int kTileThreads = 128;  // threads of a time-loop block (every launch shape)

// The last 96 bytes of sw100_patch_step (ster onwards): everything the
// set-bit walk reads, in the record's 16-byte groups.  With the dense sums
// precomputed the loop stages only these, 96-byte records instead of 128 (a
// smaller block, and lanes reading different patches spread over more
// banks).
struct PatchTail {
  float ster, cos_alt, sin_alt, kref_veg;
  double veg_cos, veg_sin;
  float yi_k, thr_sun, thr_shd;
  int32_t flags;
  float kref_sun, kref_sh, yi_l, ld_sky;
  float sun_cos, sun_sin, ls_sky;
  int32_t pad;
  double sh_cos, sh_sin;
};
constexpr int kPatchTailOffset = (int)offsetof(sw100_patch_step, ster);
static_assert(kPatchTailOffset == 32 && sizeof(PatchTail) == 96 &&
                  sizeof(sw100_patch_step) == kPatchTailOffset + sizeof(PatchTail),
              "PatchTail is the tail of sw100_patch_step");
#define SW100_TAIL_AT(f) (offsetof(PatchTail, f) + kPatchTailOffset == offsetof(sw100_patch_step, f))
static_assert(SW100_TAIL_AT(ster) && SW100_TAIL_AT(veg_cos) && SW100_TAIL_AT(yi_k) && SW100_TAIL_AT(flags) &&
                  SW100_TAIL_AT(kref_sun) && SW100_TAIL_AT(sun_cos) && SW100_TAIL_AT(sh_cos),
              "PatchTail fields sit where sw100_patch_step has them");
#undef SW100_TAIL_AT
static_assert(offsetof(sw100_patch_step, ster) % 16 == 0 && offsetof(sw100_patch_step, veg_cos) % 16 == 0 &&
                  offsetof(sw100_patch_step, yi_k) % 16 == 0 && offsetof(sw100_patch_step, kref_sun) % 16 == 0 &&
                  offsetof(sw100_patch_step, sun_cos) % 16 == 0 && offsetof(sw100_patch_step, sh_cos) % 16 == 0,
              "the walk's 16-byte groups are 16-byte aligned in the record");

struct GvfAzSmem {
  int8_t dx[SW100_MAX_GVF_STEPS];
  int8_t dy[SW100_MAX_GVF_STEPS];
  int32_t facesh_mode;
  float facesh_lo;
  float facesh_hi;
  int32_t dir_flags;
};

__device__ __forceinline__ float facesh_value(int mode, float lo, float hi, float aspect, float wallbol) {
  if (mode == 0) return ((aspect < lo || aspect >= hi) ? 1.f : 0.f) - wallbol + 1.f;
  return ((aspect > lo || aspect <= hi) ? 1.f : 0.f) * -1.f + 1.f;
}

// float32 transcendental rounded once from double
__device__ __forceinline__ float atan_r(float x) { return (float)atan((double)x); }
__device__ __forceinline__ float sin_r(float x) { return (float)sin((double)x); }
__device__ __forceinline__ float cos_r(float x) { return (float)cos((double)x); }

// cylindric_wedge (solweig.py:404-449) + NaN -> 0.5 (solweig.py:2168).
// Out of line: its double-precision atan / sin / cos are a large block of
// code run once per pixel and step, kept out of the step's loop code.
__device__ __noinline__ float cylindric_wedge(float ta, float tb, float qa) {
  const float tt = ta * tb;
  const float xa = 1.f - 2.f / tt;
  const float ha = 2.f / tt;
  const float ba = 1.f / ta;
  const float hkil = (2.f * ba) * ha;
  float ukil = 0.f;
  if (xa < 0.f) {
    const float za = sqrtf(ba * ba - (qa * qa) / 4.f);
    const float phi = atan_r(za / qa);
    const float cphi = cos_r(phi);
    const float A = (sin_r(phi) - phi * cphi) / (1.f - cphi);
    ukil = ((2.f * ba) * xa) * A;
  }
  const float ssurf = hkil + ukil;
  const float twopi_ba = 6.28318548202514648f * ba;  // float32(2 * pi) * ba
  float fsh = (twopi_ba - ssurf) / twopi_ba;
  if (fsh != fsh) fsh = 0.5f;
  return fsh;
}

// One ground-view-factor search direction (sunonsurface_2018a,
// solweig.py:155-213) for one pixel.  The reference's running minimum f is
// 0/1: it is 1 until the walk first meets a building sample and 0 from then
// on.  While f == 1 the shadow / Lup / albedo sums grow by the sample and
// tempbub is the running OR of the sunlit-wall samples; once f == 0 those
// sums add exact zeros, tempbub is frozen and tempbubwall is 1.  The wall
// sums only ever add 0 or one constant (Lwall, albedo_b), so each equals
// that constant added k times in float32, k counted here and the value
// looked up in a per-step table.  The walk therefore stops at the first
// building, and every sum is the reference's own float32 sequence.
struct GvfWalk {
  float sLup, sAlb, sNosh;   // weightsum{Lupsh, albsh, albnosh} after `second` steps
  float qLup, qAlb, qNosh;   // the same after the `first` snapshot
  int m, m2;                 // steps with tempbub == 1 / tempbubwall == 1 (all steps)
  int qm, qm2;               // the same at the snapshot
};

template <bool CHECKED>
__device__ __forceinline__ GvfWalk gvf_walk(const float4* __restrict__ G, size_t p, int r, int c, int rows,
                                            int cols, const int8_t* dx, const int8_t* dy, const int* off,
                                            float bld, int second_i, int snap_n) {
  float sLup = 0.f, sAlb = 0.f, sNosh = 0.f, qLup = 0.f, qAlb = 0.f, qNosh = 0.f;
  int tb = 0, m = 0, n0 = second_i, qm = -1;
  if (bld == 0.f) {
    n0 = 0;  // f = min(buildings, .) is 0 from the first step
  } else {
    // the sample of the last in-grid step (the reference never clears its
    // temporaries); step 0 has no shift, so it is always in the grid
    uint32_t fl = 0u;
    float tlup = 0.f, talb = 0.f, talbsh = 0.f;
    for (int n = 0; n < second_i; ++n) {
      bool load = true;
      size_t src = 0;
      if (CHECKED) {
        const int sr = r + dx[n], sc = c + dy[n];
        load = in_grid(sr, sc, rows, cols);
        src = (size_t)sr * cols + sc;
      } else {
        src = (size_t)((long long)p + off[n]);
      }
      if (load) {
        const float4 g = G[src];
        fl = __float_as_uint(g.w);
        tlup = g.y;
        talb = g.z;
        talbsh = g.z * g.x;  // albshadow = alb * shadow
      }
      if (!(fl & 1u)) {  // a building sample: f becomes 0
        n0 = n;
        break;
      }
      sLup = sLup + tlup;
      sAlb = sAlb + talbsh;
      sNosh = sNosh + talb;
      tb |= (int)((fl >> 1) & 1u);
      m += tb;
      if (n + 1 == snap_n) { qLup = sLup; qAlb = sAlb; qNosh = sNosh; qm = m; }
    }
  }
  GvfWalk W;
  W.sLup = sLup; W.sAlb = sAlb; W.sNosh = sNosh;
  const int rest = second_i - n0;  // steps with f == 0
  W.m = m + tb * rest;
  W.m2 = rest;
  if (qm < 0) {  // the snapshot lies at or after the first building
    W.qLup = sLup; W.qAlb = sAlb; W.qNosh = sNosh;
    W.qm = m + tb * (snap_n - n0);
    W.qm2 = snap_n - n0;
  } else {
    W.qLup = qLup; W.qAlb = qAlb; W.qNosh = qNosh;
    W.qm = qm;
    W.qm2 = 0;
  }
  return W;
}

// The same walk when the first building's step n0 is already known: the
// building samples depend on the buildings raster only (flag bit 0 of the
// sun-march records), so n0 is the same at every daytime step and the
// walk needs no test for it -- its n0 gathers do not wait on each other.
template <bool CHECKED>
__device__ __forceinline__ GvfWalk gvf_walk_known(const float4* __restrict__ G, size_t p, int r, int c, int rows,
                                                  int cols, const int8_t* dx, const int8_t* dy, const int* off,
                                                  int n0, int second_i, int snap_n) {
  float sLup = 0.f, sAlb = 0.f, sNosh = 0.f, qLup = 0.f, qAlb = 0.f, qNosh = 0.f;
  int tb = 0, m = 0, qm = -1;
  uint32_t fl = 0u;
  float tlup = 0.f, talb = 0.f, talbsh = 0.f;
  for (int n = 0; n < n0; ++n) {
    if (CHECKED) {
      const int sr = r + dx[n], sc = c + dy[n];
      if (in_grid(sr, sc, rows, cols)) {
        const float4 g = G[(size_t)sr * cols + sc];
        fl = __float_as_uint(g.w);
        tlup = g.y;
        talb = g.z;
        talbsh = g.z * g.x;
      }
    } else {
      const float4 g = G[(size_t)((long long)p + off[n])];
      fl = __float_as_uint(g.w);
      tlup = g.y;
      talb = g.z;
      talbsh = g.z * g.x;
    }
    sLup = sLup + tlup;
    sAlb = sAlb + talbsh;
    sNosh = sNosh + talb;
    tb |= (int)((fl >> 1) & 1u);
    m += tb;
    if (n + 1 == snap_n) { qLup = sLup; qAlb = sAlb; qNosh = sNosh; qm = m; }
  }
  GvfWalk W;
  W.sLup = sLup; W.sAlb = sAlb; W.sNosh = sNosh;
  const int rest = second_i - n0;
  W.m = m + tb * rest;
  W.m2 = rest;
  if (qm < 0) {
    W.qLup = sLup; W.qAlb = sAlb; W.qNosh = sNosh;
    W.qm = m + tb * (snap_n - n0);
    W.qm2 = snap_n - n0;
  } else {
    W.qLup = qLup; W.qAlb = qAlb; W.qNosh = qNosh;
    W.qm = qm;
    W.qm2 = 0;
  }
  return W;
}

// The walks of pixels near the grid edge (bounds-tested steps) out of line:
// few pixels take them, and keeping their code out of the per-azimuth loop
// leaves that loop's instructions in the instruction cache (2-3 % faster
// loop kernel at 500 x 500 to 2048 x 2048).
__device__ __noinline__ GvfWalk gvf_walk_edge(const float4* __restrict__ G, size_t p, int r, int c, int rows,
                                              int cols, const int8_t* dx, const int8_t* dy, const int* off,
                                              float bld, int second_i, int snap_n) {
  return gvf_walk<true>(G, p, r, c, rows, cols, dx, dy, off, bld, second_i, snap_n);
}

__device__ __noinline__ GvfWalk gvf_walk_known_edge(const float4* __restrict__ G, size_t p, int r, int c, int rows,
                                                    int cols, const int8_t* dx, const int8_t* dy, const int* off,
                                                    int n0, int second_i, int snap_n) {
  return gvf_walk_known<true>(G, p, r, c, rows, cols, dx, dy, off, n0, second_i, snap_n);
}

// x / d for a divisor shared by every pixel of a step, given rd, the
// correctly rounded float32 reciprocal of d.  Markstein's theorem (IBM J.
// Res. Dev. 34(1), 1990; Muller et al., Handbook of Floating-Point
// Arithmetic, ch. 5): q = x * rd is within one ulp of x / d, the remainder
// x - q * d is exact in one FMA, and q + r * rd rounded once is the
// correctly rounded quotient -- the IEEE float32 x / d -- for operands in the
// normal range.  Three instructions instead of a full division.
// FAST: x * rd alone (within one ulp of the quotient), for the loop variant
// whose fluxes are held to the Tmrt tolerance rather than to the
// reference's bits.
template <bool FAST = false>
__device__ __forceinline__ float div_by(float x, float d, float rd) {
  if constexpr (FAST) return __fmul_rn(x, rd);
  const float q = __fmul_rn(x, rd);
  const float r = __fmaf_rn(-q, d, x);
  return __fmaf_rn(r, rd, q);
}

// Bits of the patches q0 .. q0 + 31 that exist (n_patches of them in all).
__device__ __forceinline__ uint32_t patch_word_mask(int n_patches, int q0) {
  const int n = n_patches - q0;
  return n >= 32 ? 0xffffffffu : (n <= 0 ? 0u : ((1u << n) - 1u));
}

// Divisors of the walk epilogue, with their reciprocals.
struct StepDiv {
  float first, f1, second, s1, rfirst, rf1, rsecond, rs1;
};

// `x / d * sel + y / e * (1 - sel)` of the reference with sel in {0, 1}:
// one of the two products is an exact zero, so only one quotient is needed
// (the zero is still added, keeping the float32 result identical)
template <bool FAST = false>
__device__ __forceinline__ float pick_div(bool sel, float x, float d, float rd, float y, float e, float re) {
  if constexpr (FAST) return sel ? __fmul_rn(x, rd) : __fmul_rn(y, re);
  return sel ? (div_by(x, d, rd) + 0.f) : (0.f + div_by(y, e, re));
}

// correctly rounded float32 reciprocals of 0.9f, 18 and 9
constexpr float kR09 = 0x1.1c71c8p+0f;
constexpr float kR18 = 0x1.c71c72p-5f;
constexpr float kR9 = 0x1.c71c72p-4f;

// a float64 term added to a sum: in float64 and rounded to float32 each
// time (the reference's float32 array += float64 scalar), or kept in
// float64 (HELD: the sum is a double)
template <bool HELD, class A>
__device__ __forceinline__ void acc64(A& acc, double term) {
  if constexpr (HELD) acc = acc + term;
  else acc = add64(acc, term);
}

struct GvfSums {
  float Lup, alb, albnosh;
  float LupE, albE, albnoshE, LupS, albS, albnoshS, LupW, albW, albnoshW, LupN, albN, albnoshN;
};

// All steps of the pixels of tile (bx, by); every thread of the block calls
// it (the step tables are staged in shared memory).  With `order` (the
// site's patch order, n_order patches) the block is instead four 8 x 4
// pixel patches, warp w taking patch order[bx * 4 + w].  `Site` is SitePlanes
// (a kernel parameter) or sw100_site_planes (a batch descriptor in global
// memory): the same member names.
// KNOWN_N0: reuse each walk's first-building step after the first daytime
// step (faster for one site and for the batch with tensor-core sums; the
// in-loop-sums batch kernel, with more live registers, does not gain).
// SUMS: the four dense patch sums of each step come precomputed (the
// tensor-core product of patch_sums.cu, sums[(t * 4 + j) * npix + p], j =
// diffuse Kside, anisotropic luminance, sky longwave down, side) instead of
// the dense pass below.
template <class Site, bool KNOWN_N0, bool SUMS = false>
__device__ __forceinline__ void time_loop_tile(
    const Site& site, int rows, int cols, const sw100_time_step* __restrict__ tsteps, int n_t,
    const sw100_patch_step* __restrict__ patch_steps, int n_patches,
    const sw100_gvf_azimuth* __restrict__ gvf_az, const float4* __restrict__ gsrc, int n_day,
    float* __restrict__ state, uint32_t out_mask, float* __restrict__ outputs, int bx, int by,
    const float* __restrict__ sums = nullptr, const int32_t* __restrict__ order = nullptr, int n_order = 0) {
  // PP is filled with 16-byte vector stores: the array must be 16-byte
  // aligned (the struct itself only requires 8)
  __shared__ __align__(16) sw100_time_step P;
  using PatchRec = typename std::conditional<SUMS, PatchTail, sw100_patch_step>::type;
  __shared__ __align__(16) PatchRec PP[kMaxPatchSmem];
  __shared__ GvfAzSmem AZ[SW100_N_GVF_AZ];
  __shared__ int AZOFF[SW100_N_GVF_AZ][SW100_MAX_GVF_STEPS];  // dx * cols + dy
  // Lwall / albedo_b added k times in float32, k = 0..second (this step)
  __shared__ float REP_L[SW100_MAX_GVF_STEPS + 1], REP_A[SW100_MAX_GVF_STEPS + 1];
  // first-building step of each ground-view walk of the thread's pixel,
  // found at its first daytime step and reused at the later ones
  __shared__ uint8_t N0[SW100_N_GVF_AZ][kTileThreads];
  int n0_second = -1;  // the walk length N0 was found for (-1: not yet)
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nthr = blockDim.x * blockDim.y;
  for (int i = tid; i < SW100_N_GVF_AZ * SW100_MAX_GVF_STEPS; i += nthr) {
    const int a = i / SW100_MAX_GVF_STEPS, n = i % SW100_MAX_GVF_STEPS;
    AZ[a].dx[n] = gvf_az[a].dx[n];
    AZ[a].dy[n] = gvf_az[a].dy[n];
    AZOFF[a][n] = (int)gvf_az[a].dx[n] * cols + (int)gvf_az[a].dy[n];
  }
  if (tid < SW100_N_GVF_AZ) {
    AZ[tid].facesh_mode = gvf_az[tid].facesh_mode;
    AZ[tid].facesh_lo = gvf_az[tid].facesh_lo;
    AZ[tid].facesh_hi = gvf_az[tid].facesh_hi;
    AZ[tid].dir_flags = gvf_az[tid].dir_flags;
  }
  int c = bx * blockDim.x + threadIdx.x;
  int r = by * blockDim.y + threadIdx.y;
  if (order != nullptr) {
    const int k = bx * 4 + (tid >> 5), lane = tid & 31, pcols = (cols + 7) >> 3;
    const int pt = k < n_order ? order[k] : -1;
    const bool ok = pt >= 0 && pt < n_order;
    r = ok ? (pt / pcols) * 4 + (lane >> 3) : rows;  // rows: no pixel
    c = ok ? (pt % pcols) * 8 + (lane & 7) : cols;
  }
  const bool live = (r < rows) && (c < cols);
  const size_t npix = (size_t)rows * cols;
  const size_t p = live ? (size_t)r * cols + c : 0;

  // per-pixel statics
  float bld = 0.f, walls = 0.f, aspect = 0.f, emis = 0.f, alb = 0.f, svfbuveg = 0.f, hsvf = 0.f, tan_alfa = 0.f,
        wind = 0.f;
  // the pixel's patch-bit words (sh, vegsh, vbshvegsh cubes) live in shared
  // memory, one column per thread: registers go to the per-step work
  __shared__ uint32_t CB[3 * SW100_CUBE_WORDS][kTileThreads];
  const int ctid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int w = 0; w < 3 * SW100_CUBE_WORDS; ++w) CB[w][ctid] = 0u;
  float st[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // Tgmap1, E, S, W, N, TgOut1
  if (live) {
    bld = site.buildings[p];
    walls = site.walls[p];
    aspect = site.aspect_rad[p];
    emis = site.emis[p];
    alb = site.alb[p];
    svfbuveg = site.svfbuveg[p];
    hsvf = site.hsvf[p];
    tan_alfa = site.tan_alfa[p];
    wind = site.windcoeff[p];
#pragma unroll
    for (int w = 0; w < SW100_CUBE_WORDS; ++w) {
      CB[w][ctid] = site.bits[(0 * SW100_CUBE_WORDS + w) * npix + p];
      CB[SW100_CUBE_WORDS + w][ctid] = site.bits[(1 * SW100_CUBE_WORDS + w) * npix + p];
      CB[2 * SW100_CUBE_WORDS + w][ctid] = site.bits[(2 * SW100_CUBE_WORDS + w) * npix + p];
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) st[k] = state[k * npix + p];
  }
  const float wallbol = walls > 0.f ? 1.f : 0.f;
  const float nb = bld * -1.f + 1.f;

  for (int t = 0; t < n_t; ++t) {
    __syncthreads();
    {
      const int* s = reinterpret_cast<const int*>(&tsteps[t]);
      int* d = reinterpret_cast<int*>(&P);
      for (int i = tid; i < (int)(sizeof(sw100_time_step) / 4); i += nthr) d[i] = s[i];
      const int4* ps = reinterpret_cast<const int4*>(patch_steps + (size_t)t * n_patches);
      int4* pd = reinterpret_cast<int4*>(PP);
      // 16-byte pieces per staged record, and where the record starts in
      // the 128-byte global one
      constexpr int kPieces = (int)(sizeof(PatchRec) / 16);
      constexpr int kSkip = (int)((sizeof(sw100_patch_step) - sizeof(PatchRec)) / 16);
      const int n16 = n_patches * kPieces;
      for (int i = tid; i < n16; i += nthr) {
        const int rec = i / kPieces, piece = i - rec * kPieces;
        pd[i] = ps[rec * (kPieces + kSkip) + kSkip + piece];
      }
      if (tsteps[t].is_day) {
        const float lw = tsteps[t].lwall, ab = tsteps[t].albedo_b;
        for (int i = tid; i <= SW100_MAX_GVF_STEPS; i += nthr) {
          float sl = 0.f, sa = 0.f;
          for (int k = 0; k < i; ++k) { sl = sl + lw; sa = sa + ab; }
          REP_L[i] = sl;
          REP_A[i] = sa;
        }
      }
    }
    __syncthreads();
    if (!live) continue;

    float shadow = 0.f, Lup, LupE, LupS, LupW, LupN;
    float Kdown = 0.f, Kup = 0.f, KupE = 0.f, KupS = 0.f, KupW = 0.f, KupN = 0.f;
    float Kside = 0.f, ksideI = 0.f, albF_day = 0.f;
    // a daytime step reads its row of sun-march records (a row outside the
    // n_day rows written is treated as night: nothing outside is read)
    const bool is_day = P.is_day != 0 && (unsigned)P.day_row < (unsigned)n_day;
    if (is_day) {
      const float4* G = gsrc + (size_t)P.day_row * npix;
      const float4 own = G[p];
      shadow = own.x;
      const float lup_own = own.y;
      const float tg = ground_temperature(site, P, p);
      // ---------------- ground view factors (18 azimuths)
      GvfSums S = {};
      const int second_i = min((int)P.second, SW100_MAX_GVF_STEPS);  // walk tables hold 64 steps
      const float second = P.second;
      StepDiv D;
      D.first = P.first;
      D.second = second;
      D.f1 = P.first + 1.f;
      D.s1 = second + 1.f;
      D.rfirst = __frcp_rn(D.first);
      D.rf1 = __frcp_rn(D.f1);
      D.rsecond = __frcp_rn(D.second);
      D.rs1 = __frcp_rn(D.s1);
      // a pixel at least `second - 1` pixels from every edge never walks out
      // of the grid: its walk needs no bounds test
      const int reach = second_i - 1;
      const bool interior = r >= reach && r < rows - reach && c >= reach && c < cols - reach;
      const int first_i = (int)P.first;
      const int snap_n = min(first_i, second_i);  // snapshot after this many steps
      const bool n0_known = KNOWN_N0 && n0_second == second_i;
      for (int az = 0; az < SW100_N_GVF_AZ; ++az) {
        GvfWalk W;
        if (n0_known) {
          const int n0 = N0[az][ctid];
          W = interior
              ? gvf_walk_known<false>(G, p, r, c, rows, cols, AZ[az].dx, AZ[az].dy, AZOFF[az], n0, second_i, snap_n)
              : gvf_walk_known_edge(G, p, r, c, rows, cols, AZ[az].dx, AZ[az].dy, AZOFF[az], n0, second_i, snap_n);
        } else {
          W = interior
              ? gvf_walk<false>(G, p, r, c, rows, cols, AZ[az].dx, AZ[az].dy, AZOFF[az], bld, second_i, snap_n)
              : gvf_walk_edge(G, p, r, c, rows, cols, AZ[az].dx, AZ[az].dy, AZOFF[az], bld, second_i, snap_n);
          if (KNOWN_N0) N0[az][ctid] = (uint8_t)(second_i - W.m2);
        }
        // the reference's weight sums
        const float wwall = (float)W.m;
        float wLwall = REP_L[W.m], walbwall = REP_A[W.m];
        const float walbwallnosh = REP_A[W.m2];
        const float s_wall = (float)W.qm, s_Lwall = REP_L[W.qm], s_albwall = REP_A[W.qm];
        const float s_albwallnosh = REP_A[W.qm2];
        const bool wsi_f = s_wall > 0.f, wi_f = s_albwallnosh > 0.f;
        const bool wsi_s = wwall > 0.f, wi_s = walbwallnosh > 0.f;
        const float facesh = facesh_value(AZ[az].facesh_mode, AZ[az].facesh_lo, AZ[az].facesh_hi, aspect, wallbol);
        float keep = ((wwall == second) ? 1.f : 0.f) - facesh;
        if (keep == -1.f) keep = 0.f;
        const bool kz = keep == 1.f;
        if (kz) { wLwall = 0.f; walbwall = 0.f; }
        const float gLup1 = pick_div<SUMS>(wsi_f, s_Lwall + W.qLup, D.f1, D.rf1, W.qLup, D.first, D.rfirst);
        const float gLup2 = pick_div<SUMS>(wsi_s, wLwall + W.sLup, D.s1, D.rs1, W.sLup, D.second, D.rsecond);
        const float galb1 = pick_div<SUMS>(wsi_f, s_albwall + W.qAlb, D.f1, D.rf1, W.qAlb, D.first, D.rfirst);
        const float galb2 = pick_div<SUMS>(wsi_s, walbwall + W.sAlb, D.s1, D.rs1, W.sAlb, D.second, D.rsecond);
        const float gan1 = pick_div<SUMS>(wi_f, s_albwallnosh + W.qNosh, D.f1, D.rf1, W.qNosh, D.first, D.rfirst);
        const float gan2 = pick_div<SUMS>(wi_s, walbwallnosh + W.sNosh, D.second, D.rsecond, W.sNosh, D.second, D.rsecond);
        const float gLup = div_by<SUMS>(gLup1 * 0.5f + gLup2 * 0.4f, 0.9f, kR09) + lup_own * nb;
        const float galb = div_by<SUMS>(galb1 * 0.5f + galb2 * 0.4f, 0.9f, kR09) + (alb * nb) * shadow;
        const float gan = div_by<SUMS>(gan1 * 0.5f + gan2 * 0.4f, 0.9f, kR09) * bld + alb * nb;
        S.Lup = S.Lup + gLup;
        S.alb = S.alb + galb;
        S.albnosh = S.albnosh + gan;
        const int df = AZ[az].dir_flags;
        if (df & 1) { S.LupE = S.LupE + gLup; S.albE = S.albE + galb; S.albnoshE = S.albnoshE + gan; }
        if (df & 2) { S.LupS = S.LupS + gLup; S.albS = S.albS + galb; S.albnoshS = S.albnoshS + gan; }
        if (df & 4) { S.LupW = S.LupW + gLup; S.albW = S.albW + galb; S.albnoshW = S.albnoshW + gan; }
        if (df & 8) { S.LupN = S.LupN + gLup; S.albN = S.albN + galb; S.albnoshN = S.albnoshN + gan; }
      }
      n0_second = second_i;
      const float lup_air = (P.sbc * emis) * P.ta4;
      const float gvfLup = div_by<SUMS>(S.Lup, 18.f, kR18) + lup_air;
      const float gvfalb = div_by<SUMS>(S.alb, 18.f, kR18), gvfalbnosh = div_by<SUMS>(S.albnosh, 18.f, kR18);
      const float gvfLupE = div_by<SUMS>(S.LupE, 9.f, kR9) + lup_air, gvfLupS = div_by<SUMS>(S.LupS, 9.f, kR9) + lup_air;
      const float gvfLupW = div_by<SUMS>(S.LupW, 9.f, kR9) + lup_air, gvfLupN = div_by<SUMS>(S.LupN, 9.f, kR9) + lup_air;
      const float gvfalbE = div_by<SUMS>(S.albE, 9.f, kR9), gvfalbS = div_by<SUMS>(S.albS, 9.f, kR9);
      const float gvfalbW = div_by<SUMS>(S.albW, 9.f, kR9), gvfalbN = div_by<SUMS>(S.albN, 9.f, kR9);
      const float ganE = div_by<SUMS>(S.albnoshE, 9.f, kR9), ganS = div_by<SUMS>(S.albnoshS, 9.f, kR9);
      const float ganW = div_by<SUMS>(S.albnoshW, 9.f, kR9), ganN = div_by<SUMS>(S.albnoshN, 9.f, kR9);
      // ---------------- thermal lag (state in registers)
      const float tgtemp = tg * shadow + P.ta32;
      const float g0[6] = {gvfLup, gvfLupE, gvfLupS, gvfLupW, gvfLupN, tgtemp};
      float lagged[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        if (P.tw_first) st[k] = g0[k];
        const float v = g0[k] * P.tw_a + st[k] * P.tw_b;
        if (P.tw_mode) st[k] = v;
        lagged[k] = v;
      }
      Lup = lagged[0]; LupE = lagged[1]; LupS = lagged[2]; LupW = lagged[3]; LupN = lagged[4];
      // ---------------- shortwave
      const float fsh = cylindric_wedge(tan_alfa, P.tan_beta, P.qa);
      const float albF = (P.albedo_b * (1.f - svfbuveg)) * (P.radG * (1.f - fsh) + P.radD * fsh);
      const float kup_b = P.radD * svfbuveg + albF;
      Kup = (gvfalb * P.radI) * P.sin_alt + kup_b * gvfalbnosh;
      KupE = (gvfalbE * P.radI) * P.sin_alt + kup_b * ganE;
      KupS = (gvfalbS * P.radI) * P.sin_alt + kup_b * ganS;
      KupW = (gvfalbW * P.radI) * P.sin_alt + kup_b * ganW;
      KupN = (gvfalbN * P.radI) * P.sin_alt + kup_b * ganN;
      ksideI = (shadow * P.radI) * P.cos_alt;
      albF_day = albF;
    } else {
      Lup = (P.sbc * emis) * pow4f(P.night_lup_base);
      LupE = LupS = LupW = LupN = Lup;
    }
    // ---------------- 153-patch sums: Kside (day) and Lcyl
    // (solweig.py:683-724, 1514-1633).  Every sum is its own accumulator fed
    // in patch order, so the patches are visited per sum: one dense pass for
    // the sums that take (almost) every patch, and ascending set-bit walks
    // of a per-pixel mask for the sums that take few.
    float ksideD = 0.f, kref_sun = 0.f, kref_sh = 0.f, kref_veg = 0.f, anilum = 0.f;
    float ld_sky = 0.f, ld_veg = 0.f, ld_sh = 0.f, ld_sun = 0.f, ld_ref = 0.f;
    float ls_sky = 0.f, ls_veg = 0.f, ls_sh = 0.f, ls_sun = 0.f, ls_ref = 0.f;
    // The float64 increments (vegetation and shaded-wall longwave): the
    // reference adds each to a float32 sum in float64 and rounds (add64).
    // With the dense sums from the tensor cores the fluxes are already held
    // to the Tmrt tolerance rather than to the reference's bits, and these
    // four sums stay in float64 until the end: no conversion per term.
    using Acc64 = typename std::conditional<SUMS, double, float>::type;
    Acc64 ls_veg_a = 0, ld_veg_a = 0, ls_sh_a = 0, ld_sh_a = 0;
    const bool day = is_day;
    if (SUMS) {
      const float* sp = sums + (size_t)t * 4 * npix + p;
      if (day) {
        ksideD = sp[0];
        anilum = sp[npix];
      }
      ld_sky = sp[2 * npix];
      ls_sky = sp[3 * npix];
    }
    // dense: sky-visible longwave (sh == 1 & vegsh == 1); by day the diffuse
    // Kside term and the anisotropic luminance, indexed by (sh, vegsh)
    if constexpr (!SUMS) {
#pragma unroll
    for (int w = 0; w < SW100_CUBE_WORDS; ++w) {
      const int q0 = w * 32;
      const int nq = min(32, n_patches - q0);
      const uint32_t sw = CB[w][ctid], vw = CB[SW100_CUBE_WORDS + w][ctid];
      if (day) {
        for (int j = 0; j < nq; ++j) {
          const sw100_patch_step& Q = PP[q0 + j];
          // the (sh, vegsh) code indexes the patch's four increments: lanes
          // read different words of one 16-byte group, no bank conflict
          const int code = (int)((sw >> j) & 1u) * 2 + (int)((vw >> j) & 1u);
          ksideD = ksideD + Q.kside_d[code];
          anilum = anilum + Q.anilum[code];
          if (code == 3) { ld_sky = ld_sky + Q.ld_sky; ls_sky = ls_sky + Q.ls_sky; }
        }
      } else {
        for (int j = 0; j < nq; ++j) {
          if ((sw >> j) & (vw >> j) & 1u) {
            const sw100_patch_step& Q = PP[q0 + j];
            ld_sky = ld_sky + Q.ld_sky;
            ls_sky = ls_sky + Q.ls_sky;
          }
        }
      }
    }
    }
    // One ascending set-bit walk over the reflected-longwave patches
    // (solweig.py:1613-1633, temp_sh = (sh == 0) | (vegsh == 0) |
    // (vbshvegsh == 0)), a superset of the vegetation-facing patches
    // (vegsh == 0 or vbshvegsh == 0: vegetation longwave in float64 adds and
    // by day the vegetation-reflected Kside) and of the wall-facing patches
    // ((1 - sh) * vbshvegsh == 1: sunlit / shaded wall terms split by the
    // shaded_or_sunlit predicate).  Each accumulator still receives its
    // terms in patch order.
    const float refl = (((ld_sky + Lup) * P.refl_k) * 0.5f) / 3.14159274101257324f;
    float ref_c = 0.f, ref_s = 0.f;   // sums of ster * cos / sin over the reflecting patches (SUMS)
#pragma unroll
    for (int w = 0; w < SW100_CUBE_WORDS; ++w) {
      const int q0 = w * 32;
      const uint32_t bsh = CB[w][ctid], bveg = CB[SW100_CUBE_WORDS + w][ctid];
      const uint32_t bvb = CB[2 * SW100_CUBE_WORDS + w][ctid];
      const uint32_t pm = patch_word_mask(n_patches, q0);
      const uint32_t mveg = (~bveg | (~bvb & ~site.single_step[w])) & pm;
      const uint32_t mwall = ~bsh & bvb & pm;
      uint32_t m = (~bsh | mveg) & pm;
      while (m) {
        const int j = __ffs(m) - 1;
        m &= m - 1u;
        const uint32_t bit = 1u << j;
        const PatchRec& Q = PP[q0 + j];
        // the record's 16-byte groups (16-byte aligned in PP): one shared
        // load each
        const float4 R = *reinterpret_cast<const float4*>(&Q.ster);   // ster, cos_alt, sin_alt, kref_veg
        if (mveg & bit) {
          const double2 V = *reinterpret_cast<const double2*>(&Q.veg_cos);
          acc64<SUMS>(ls_veg_a, V.x);
          acc64<SUMS>(ld_veg_a, V.y);
          if (day) kref_veg = kref_veg + R.w;
        }
        if (mwall & bit) {
          const float4 W = *reinterpret_cast<const float4*>(&Q.yi_k);       // yi_k, thr_sun, thr_shd, flags
          const float4 K = *reinterpret_cast<const float4*>(&Q.kref_sun);   // kref_sun, kref_sh, yi_l, ld_sky
          if (day) {
            const float td = hsvf + W.x;
            if (td < W.y) kref_sun = kref_sun + K.x;
            if (td > W.z) kref_sh = kref_sh + K.y;
          }
          const double2 H = *reinterpret_cast<const double2*>(&Q.sh_cos);
          if (__float_as_int(W.w) & 1) {
            const float td = hsvf + K.z;
            if (td < W.y) {
              const float2 U = *reinterpret_cast<const float2*>(&Q.sun_cos);
              ls_sun = ls_sun + U.x;
              ld_sun = ld_sun + U.y;
            }
            if (td > W.z) { acc64<SUMS>(ls_sh_a, H.x); acc64<SUMS>(ld_sh_a, H.y); }
          } else {
            acc64<SUMS>(ls_sh_a, H.x);
            acc64<SUMS>(ld_sh_a, H.y);
          }
        }
        if constexpr (SUMS) {   // refl * sum(ster * cos) once, below
          ref_c = __fmaf_rn(R.x, R.y, ref_c);
          ref_s = __fmaf_rn(R.x, R.z, ref_s);
        } else {
          const float rs = refl * R.x;
          ls_ref = ls_ref + rs * R.y;
          ld_ref = ld_ref + rs * R.z;
        }
      }
    }
    if constexpr (SUMS) {
      ls_ref = refl * ref_c;
      ld_ref = refl * ref_s;
    }
    if (day) {
      Kside = (((ksideI + ksideD) + kref_sun) + kref_sh) + kref_veg;
      const float dRad = anilum * P.radD;
      Kdown = ((P.radI * shadow) * P.sin_alt + dRad) + albF_day;
    }
    ls_veg = (float)ls_veg_a; ld_veg = (float)ld_veg_a; ls_sh = (float)ls_sh_a; ld_sh = (float)ld_sh_a;
    const float Lside = (((ls_sky + ls_veg) + ls_sh) + ls_sun) + ls_ref;
    const float Ldown = (((ld_sky + ld_veg) + ld_sh) + ld_sun) + ld_ref;
    // ---------------- Tmrt (cyl == 1, anisotropic sky)
    const float Knorth = KupN * 0.5f, Keast = KupE * 0.5f, Ksouth = KupS * 0.5f, Kwest = KupW * 0.5f;
    const float Lnorth = LupN * 0.5f, Least = LupE * 0.5f, Lsouth = LupS * 0.5f, Lwest = LupW * 0.5f;
    const float sstr = P.absK * (Kside * P.Fcyl + (Kdown + Kup) * P.Fup + (((Knorth + Keast) + Ksouth) + Kwest) * P.Fside) +
                       P.absL * ((Ldown + Lup) * P.Fup + Lside * P.Fcyl + (((Lnorth + Least) + Lsouth) + Lwest) * P.Fside);
    const float tmrt = sqrtf(sqrtf(sstr / P.absl_sbc)) - 273.2f;
    // ---------------- outputs
    float* o = outputs + (size_t)t * npix + p;
    const size_t blk = (size_t)n_t * npix;
    int slot = 0;
    if (out_mask & SW100_OUT_UTCI) {
      float u;
      if (!(bld == 1.f)) {
        u = __int_as_float(0x7fc00000);
      } else {
        float va = wind * P.ws32;
        va = (va < 0.15f) ? 0.15f : va;
        if (P.ta_mat <= -999.f || P.rh32 <= -999.f || va <= -999.f || tmrt <= -999.f) u = -999.f;
        else u = utci_series_step(P.utci_k, P.utci_pa, P.ta_mat, va, tmrt - P.ta_mat);
      }
      o[slot++ * blk] = u;
    }
    if (out_mask & SW100_OUT_TMRT) o[slot++ * blk] = tmrt;
    if (out_mask & SW100_OUT_KUP) o[slot++ * blk] = Kup;
    if (out_mask & SW100_OUT_KDOWN) o[slot++ * blk] = Kdown;
    if (out_mask & SW100_OUT_LUP) o[slot++ * blk] = Lup;
    if (out_mask & SW100_OUT_LDOWN) o[slot++ * blk] = Ldown;
    if (out_mask & SW100_OUT_SHADOW) o[slot++ * blk] = shadow;
  }
  if (live) {
#pragma unroll
    for (int k = 0; k < 6; ++k) state[k * npix + p] = st[k];
  }
}

__global__ void __launch_bounds__(kTileThreads, 6) time_loop_kernel(
    SitePlanes site, int rows, int cols, const sw100_time_step* __restrict__ tsteps, int n_t,
    const sw100_patch_step* __restrict__ patch_steps, int n_patches,
    const sw100_gvf_azimuth* __restrict__ gvf_az, const float4* __restrict__ gsrc, int n_day,
    float* __restrict__ state, uint32_t out_mask, float* __restrict__ outputs) {
  time_loop_tile<SitePlanes, true>(site, rows, cols, tsteps, n_t, patch_steps, n_patches, gvf_az, gsrc, n_day, state,
                                   out_mask, outputs, blockIdx.x, blockIdx.y, nullptr, site.patch_order,
                                   site.n_patch_order);
}

// The same time loop with the dense patch sums precomputed on the tensor
// cores (patch_sums_tc_kernel).
__global__ void __launch_bounds__(kTileThreads, 6) time_loop_sums_kernel(
    SitePlanes site, int rows, int cols, const sw100_time_step* __restrict__ tsteps, int n_t,
    const sw100_patch_step* __restrict__ patch_steps, int n_patches,
    const sw100_gvf_azimuth* __restrict__ gvf_az, const float4* __restrict__ gsrc, int n_day,
    float* __restrict__ state, uint32_t out_mask, float* __restrict__ outputs, const float* __restrict__ sums) {
  time_loop_tile<SitePlanes, true, true>(site, rows, cols, tsteps, n_t, patch_steps, n_patches, gvf_az, gsrc, n_day,
                                         state, out_mask, outputs, blockIdx.x, blockIdx.y, sums, site.patch_order,
                                         site.n_patch_order);
}

// Ground-view walk work of the loops' 8 x 4 pixel patches, one warp per
// patch: per azimuth the longest walk of its pixels to the first building
// sample in the grid (at most `second` steps; 0 for a building pixel), as
// gvf_walk stops, summed over the 18 azimuths.  The samples are read four
// steps at a time (independent loads in flight, one test per group).
__global__ void __launch_bounds__(128) walk_work_kernel(const float* __restrict__ buildings, int rows, int cols,
                                                         const sw100_gvf_azimuth* __restrict__ gvf, int second,
                                                         int32_t* __restrict__ work, int n_patch) {
  const int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (k >= n_patch) return;  // whole warps: blocks of 128 threads
  const int pcols = (cols + 7) >> 3;
  const int r = (k / pcols) * 4 + (lane >> 3), c = (k % pcols) * 8 + (lane & 7);
  const bool live = r < rows && c < cols;
  const bool ground = live && buildings[(size_t)r * cols + c] != 0.f;
  int total = 0;
  for (int az = 0; az < SW100_N_GVF_AZ; ++az) {
    int n0 = ground ? second : 0;
    for (int n = 0; ground && n < second && n0 == second; n += 4) {
      float v[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int m = n + j;
        v[j] = 1.f;
        if (m < second) {
          const int sr = r + gvf[az].dx[m], sc = c + gvf[az].dy[m];
          if (in_grid(sr, sc, rows, cols)) v[j] = buildings[(size_t)sr * cols + sc];
        }
      }
#pragma unroll
      for (int j = 3; j >= 0; --j)
        if (v[j] == 0.f) n0 = n + j;  // the first building of the group wins
    }
    total += __reduce_max_sync(0xffffffffu, n0);
  }
  if (lane == 0) work[k] = total;
}

// The time loop of every site of a batch, tiles taken in list order.
__global__ void __launch_bounds__(kTileThreads, 6) time_loop_batch_kernel(const sw100_batch_site* __restrict__ sites,
                                                                 const sw100_tile* __restrict__ tiles, int n_tiles) {
  for (int i = blockIdx.x; i < n_tiles; i += gridDim.x) {
    const sw100_tile T = tiles[i];
    const sw100_batch_site& S = sites[T.site];
    __syncthreads();  // the previous tile is done with the shared tables
    time_loop_tile<sw100_site_planes, false>(S.site, S.rows, S.cols, S.series.steps, S.series.n_t, S.series.patch, S.series.n_patches,
                   S.series.gvf, reinterpret_cast<const float4*>(S.gsrc), S.series.n_day, S.state, S.out_mask,
                   S.outputs, T.tx,
                   T.ty);
  }
}

// The same with each site's dense patch sums precomputed (S.sums).
__global__ void __launch_bounds__(kTileThreads, 6) time_loop_batch_sums_kernel(
    const sw100_batch_site* __restrict__ sites, const sw100_tile* __restrict__ tiles, int n_tiles) {
  for (int i = blockIdx.x; i < n_tiles; i += gridDim.x) {
    const sw100_tile T = tiles[i];
    const sw100_batch_site& S = sites[T.site];
    __syncthreads();  // the previous tile is done with the shared tables
    time_loop_tile<sw100_site_planes, true, true>(S.site, S.rows, S.cols, S.series.steps, S.series.n_t,
                                                   S.series.patch, S.series.n_patches, S.series.gvf,
                                                   reinterpret_cast<const float4*>(S.gsrc), S.series.n_day, S.state,
                                                   S.out_mask, S.outputs, T.tx, T.ty, S.sums);
  }
}

}  // namespace sw100
