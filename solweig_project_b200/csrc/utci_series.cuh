// UTCI in the reference's own float32 evaluation (solweig_gpu/calculate_utci.py:
// 259-330): the saturation vapour pressure chain, then the running float32 sum
// `UTCI = Ta + t_0 + t_1 + ... + t_209` of the 210-term 6th-order regression
// (Broede et al. 2012) in the order the reference writes it, every term a
// left-to-right float32 product `c * Ta^a * va^b * D^c * Pa^d` with factors of
// power 0 left out.
//
// Powers follow torch's float32 pow on a python-int exponent: x^2 = x * x and
// x^3 = (x * x) * x as float32 products; x^4..x^6 are the correctly rounded
// power (a float64 product chain rounded once to float32; torch's vector pow
// differs from that in ~2% of lanes by one ulp).  log / exp of the vapour
// pressure chain are likewise float64 rounded once to float32.  The sum is
// ill-conditioned for hot, windy inputs (partial sums reach ~2e4 while the
// result is ~50), so a one-ulp difference in one of those inputs moves the
// result by up to ulp(largest partial sum); elsewhere the value is bit-exact.
//
// The term list is generated from data/utci_terms.json into utci_series.inc
// as SW_UTCI_TERM(j, pt, pv, pd, pp, c) lines.
#pragma once

#include <cstdint>

namespace sw100 {

// x^p, p in 1..6, as torch evaluates a float32 tensor ** int
__host__ __device__ __forceinline__ float utci_pow(float x, int p) {
  if (p == 1) return x;
  if (p == 2) return x * x;
  if (p == 3) return (x * x) * x;
  const double d = x, d2 = d * d, d4 = d2 * d2;
  if (p == 4) return (float)d4;
  if (p == 5) return (float)(d4 * d);
  return (float)(d4 * d2);
}

// powers[1..6] of x (powers[0] unused)
__host__ __device__ __forceinline__ void utci_powers(float x, float* powers) {
#pragma unroll
  for (int p = 1; p <= 6; ++p) powers[p] = utci_pow(x, p);
}

// Pa = es(Ta) * RH / 100 / 10 in kPa (calculate_utci.py:273-282)
__device__ __forceinline__ float utci_vapour_pressure(float ta, float rh) {
  const float tk = ta + 273.15f;
  float es = 2.7150305f * (float)log((double)tk);
  es = es + -2.8365744E3f * (1.0f / (tk * tk));
  es = es + -6.028076559E3f * (1.0f / tk);
  es = es + 1.954263612E1f * 1.0f;
  es = es + -2.737830188E-2f * tk;
  es = es + 1.6261698E-5f * (tk * tk);
  es = es + 7.0229056E-10f * ((tk * tk) * tk);
  es = es + -1.8680009E-13f * utci_pow(tk, 4);
  es = (float)exp((double)es) * 0.01f;
  return ((es * rh) / 100.0f) / 10.0f;
}

// The running sum with every factor evaluated here (standalone UTCI).
__device__ __forceinline__ float utci_series(float ta, float va, float d, float pa) {
  float T[7], V[7], Dp[7], Pp[7];
  utci_powers(ta, T);
  utci_powers(va, V);
  utci_powers(d, Dp);
  utci_powers(pa, Pp);
  float acc = ta;
#define SW_UTCI_TERM(j, pt, pv, pd, pp, c)  \
  {                                         \
    float t_ = (pt) ? (c) * T[(pt)] : (c);  \
    if (pv) t_ = t_ * V[(pv)];              \
    if (pd) t_ = t_ * Dp[(pd)];             \
    if (pp) t_ = t_ * Pp[(pp)];             \
    acc = acc + t_;                         \
  }
#include "utci_series.inc"
#undef SW_UTCI_TERM
  return acc;
}

// The same sum for a step whose Ta and Pa are shared by every pixel: k[j] is
// c_j * Ta^pt_j (c_j where pt_j == 0) in float32 and pa[p - 1] = Pa^p, both
// tabulated on the host with the arithmetic above.
__device__ __forceinline__ float utci_series_step(const float* k, const float* pa, float ta, float va, float d) {
  float V[7], Dp[7];
  utci_powers(va, V);
  utci_powers(d, Dp);
  float acc = ta;
#define SW_UTCI_TERM(j, pt, pv, pd, pp, c) \
  {                                        \
    float t_ = k[(j)];                     \
    if (pv) t_ = t_ * V[(pv)];             \
    if (pd) t_ = t_ * Dp[(pd)];            \
    if (pp) t_ = t_ * pa[(pp) - 1];        \
    acc = acc + t_;                        \
  }
#include "utci_series.inc"
#undef SW_UTCI_TERM
  return acc;
}

}  // namespace sw100
