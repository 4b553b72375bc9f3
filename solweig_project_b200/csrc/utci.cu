// Standalone UTCI (reference solweig_gpu/calculate_utci.py:259-330) on
// float32 arrays: -999 where any input is <= -999, otherwise the reference's
// float32 evaluation (utci_series.cuh) of each element.
#include <cmath>

#include "sw_common.cuh"
#include "utci_series.cuh"

namespace sw100 {

__global__ void utci_kernel(const float* __restrict__ ta, const float* __restrict__ rh, const float* __restrict__ tmrt,
                            const float* __restrict__ va, int64_t n, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float t = ta[i], h = rh[i], m = tmrt[i], v = va[i];
    if (t <= -999.f || h <= -999.f || v <= -999.f || m <= -999.f) {
      out[i] = -999.f;
      continue;
    }
    out[i] = utci_series(t, v, m - t, utci_vapour_pressure(t, h));
  }
}

// UTCI-only recompute of whole steps (utci_process.py:1093-1196): for step
// k, UTCI of (Ta_mat, RH, the stored Tmrt plane, va = max(windcoeff * Ws,
// 0.15)) from the step's table, NaN where buildings != 1.  The same
// arithmetic as the time loop's UTCI tail.
__global__ void utci_steps_kernel(const sw100_time_step* __restrict__ steps, int n_steps,
                                  const float* __restrict__ tmrt, const float* __restrict__ buildings,
                                  const float* __restrict__ windcoeff, int64_t npix, float* __restrict__ out) {
  __shared__ __align__(16) sw100_time_step P;
  for (int k = blockIdx.y; k < n_steps; k += gridDim.y) {
    __syncthreads();
    {
      const int* s = reinterpret_cast<const int*>(&steps[k]);
      int* d = reinterpret_cast<int*>(&P);
      for (int i = threadIdx.x; i < (int)(sizeof(sw100_time_step) / 4); i += blockDim.x) d[i] = s[i];
    }
    __syncthreads();
    const float* tm = tmrt + (size_t)k * npix;
    float* o = out + (size_t)k * npix;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npix; i += (int64_t)gridDim.x * blockDim.x) {
      float u;
      if (!(buildings[i] == 1.f)) {
        u = __int_as_float(0x7fc00000);
      } else {
        const float t = tm[i];
        float va = (windcoeff ? windcoeff[i] : 1.f) * P.ws32;
        va = (va < 0.15f) ? 0.15f : va;
        if (P.ta_mat <= -999.f || P.rh32 <= -999.f || va <= -999.f || t <= -999.f) u = -999.f;
        else u = utci_series_step(P.utci_k, P.utci_pa, P.ta_mat, va, t - P.ta_mat);
      }
      o[i] = u;
    }
  }
}

}  // namespace sw100
