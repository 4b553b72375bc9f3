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

// Read-only cached load of one march step (16 bytes).
__device__ __forceinline__ sw100_step load_step(const sw100_step* p) {
  const int4 v = __ldg(reinterpret_cast<const int4*>(p));
  sw100_step s;
  s.dx = v.x;
  s.dy = v.y;
  s.dz = __int_as_float(v.z);
  s.pad = 0;
  return s;
}

}  // namespace sw100
