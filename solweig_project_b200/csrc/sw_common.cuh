// Shared device helpers for the sm_100a SOLWEIG kernels.
//
// Bit parity rules (the reference evaluates plane arithmetic as float32 torch
// tensor ops, one rounding per operation): every kernel of this library is
// compiled with --fmad=false so that no multiply-add is contracted, and the
// comparisons reproduce torch's NaN semantics where the reference relies on
// them.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "solweig_b200.h"

namespace sw100 {

// torch.maximum / torch.max(a, b): NaN propagates, on ties the second
// operand wins (ATen's `a > b || isnan(a) ? a : b`).
__device__ __forceinline__ float tmax(float a, float b) { return (a > b || a != a) ? a : b; }
// torch.minimum
__device__ __forceinline__ float tmin(float a, float b) { return (a < b || a != a) ? a : b; }

__device__ __forceinline__ bool in_grid(int r, int c, int rows, int cols) {
  return (unsigned)r < (unsigned)rows && (unsigned)c < (unsigned)cols;
}

// x**4 rounded once from double (the reference's float32 pow is within one
// ulp of this).
__device__ __forceinline__ float pow4f(float x) {
  double d = (double)x;
  d = d * d;
  return (float)(d * d);
}

// `f32 += f64-valued term` as torch does for an in-place add of a float64
// plane into a float32 plane: add in double, round once.
__device__ __forceinline__ float add64(float acc, double term) { return (float)((double)acc + term); }

struct Single5 {
  uint32_t w[SW100_CUBE_WORDS];
};

// +0 or a positive number (+inf included); false for -0, negatives and NaN.
// The march shortcuts that stop or skip steps require their thresholds to
// be non-negative so that an out-of-grid zero source changes nothing, and
// exclude -0 so that no later +0 source would have replaced a -0 maximum.
__device__ __forceinline__ bool nonneg(float x) { return __float_as_uint(x) <= 0x7f800000u; }

// Coarse bound on the march sources for skipping steps: m[b] is the largest
// of dsm, vegdsm and vegdsm2 over the 8 x 8 cell block b and its eight
// neighbours (row-major, ccol blocks per row), NaN when any of them is NaN.
// Under SW100_STEP_SKIP8 at step k, steps k .. k+7 move at most one cell per
// axis each and so stay inside the 3 x 3 blocks around step k's cell; with
// dz not decreasing, m - dz(k) bounds every source height minus drop they
// compute.  m == nullptr: no skipping.
struct SkipMap {
  const float* m;
  int ccol;
};

__device__ __forceinline__ float skip_bound(const SkipMap& s, int r, int c) {
  return __ldg(&s.m[(size_t)(r >> 3) * s.ccol + (c >> 3)]);
}

// Read-only cached load of one march step (16 bytes).
__device__ __forceinline__ sw100_step load_step(const sw100_step* p) {
  const int4 v = __ldg(reinterpret_cast<const int4*>(p));
  sw100_step s;
  s.dx = v.x;
  s.dy = v.y;
  s.dz = __int_as_float(v.z);
  s.flags = v.w;
  return s;
}

}  // namespace sw100
