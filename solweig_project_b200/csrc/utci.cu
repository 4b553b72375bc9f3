// Standalone UTCI (reference solweig_gpu/calculate_utci.py:259-330): the
// saturation vapour pressure from Ta (7-term + log form), then the 210-term
// 6th-order regression of Broede et al. (2012), evaluated in float64 from
// per-variable power tables.  The term table is generated at build time from
// solweig_project_b200/data/utci_terms.json (utci_terms.inc).
#include <cmath>

#include "sw_common.cuh"

namespace sw100 {

struct UtciTerm {
  double c;
  int8_t pt, pv, pd, pp;
};

__constant__ UtciTerm kUtciTerms[210] = {
#include "utci_terms.inc"
};

__global__ void utci_kernel(const float* __restrict__ ta, const float* __restrict__ rh, const float* __restrict__ tmrt,
                            const float* __restrict__ va, int64_t n, float* __restrict__ out) {
  const double g[8] = {-2.8365744E3, -6.028076559E3, 1.954263612E1, -2.737830188E-2,
                       1.6261698E-5, 7.0229056E-10, -1.8680009E-13, 2.7150305};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float t = ta[i], h = rh[i], m = tmrt[i], v = va[i];
    if (t <= -999.f || h <= -999.f || v <= -999.f || m <= -999.f) {
      out[i] = -999.f;
      continue;
    }
    const double tk = (double)(t + 273.15f);
    double es = g[7] * log(tk);
    for (int k = 0; k < 7; ++k) es += g[k] * pow(tk, (double)(k - 2));
    es = exp(es) * 0.01;
    const double pa = es * (double)h / 100.0 / 10.0;
    const double D = (double)(m - t);
    double pT[7], pV[7], pD[7], pP[7];
    pT[0] = pV[0] = pD[0] = pP[0] = 1.0;
    for (int k = 1; k < 7; ++k) {
      pT[k] = pT[k - 1] * (double)t;
      pV[k] = pV[k - 1] * (double)v;
      pD[k] = pD[k - 1] * D;
      pP[k] = pP[k - 1] * pa;
    }
    double acc = (double)t;
    for (int k = 0; k < 210; ++k) {
      const UtciTerm& T = kUtciTerms[k];
      acc += T.c * pT[T.pt] * pV[T.pv] * pD[T.pd] * pP[T.pp];
    }
    out[i] = (float)acc;
  }
}

}  // namespace sw100
