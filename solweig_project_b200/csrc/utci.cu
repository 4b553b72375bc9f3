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

}  // namespace sw100
