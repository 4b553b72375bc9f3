// Site preparation: the per-pixel rasters the chain derives from its inputs,
// on the device, in one pass.
//
// Reference: utci_process.py:667-681 and :1377-1385 (march rasters: canopy
// clipped at 0, vegdem / vegdem2, bush, vegdsm / vegdsm2 zeroed where equal to
// the DSM, buildings from dsm - dem < 2, amaxvalue), :733-766 with
// Tgmaps_v1.py:15-53 (land-cover cleaning and the per-class TgK, Tstart,
// albedo, emissivity) and solweig.py:2083 (wall aspect in radians).  Every
// value is the reference's float32 operation sequence rounded one operation
// at a time (--fmad=false), so the planes equal the host computation bit for
// bit; the maxima the host needs (amaxvalue, the march bound, the bush flag)
// come back as order-preserving integer keys reduced with atomics.
#include "sw_common.cuh"

namespace sw100 {

// Order-preserving key of a non-NaN float: larger float, larger key
// (-0 below +0); 0 is no float's key.
__device__ __forceinline__ uint32_t order_key(float x) {
  const uint32_t u = __float_as_uint(x);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

struct PrepAcc {
  uint32_t key[SW100_N_SITE_STATS];
  uint32_t nan_mask, nonfinite, codes, bad;
};

__device__ __forceinline__ void acc_max(PrepAcc& A, int s, float x) {
  if (x != x) A.nan_mask |= 1u << s;
  else A.key[s] = max(A.key[s], order_key(x));
}

__global__ void __launch_bounds__(256) prepare_site_kernel(
    const float* __restrict__ dsm, const float* __restrict__ trees, const float* __restrict__ dem,
    const float* __restrict__ aspect_deg, const float* __restrict__ landcover, sw100_class_table classes,
    size_t npix, float* __restrict__ vegdsm,
    float* __restrict__ vegdsm2, float* __restrict__ bush, float* __restrict__ buildings,
    float* __restrict__ aspect_rad, float* __restrict__ tgk, float* __restrict__ tstart, float* __restrict__ alb,
    float* __restrict__ emis, uint8_t* __restrict__ class_idx, sw100_site_stats* __restrict__ stats) {
  __shared__ sw100_class_table T;
  __shared__ PrepAcc B;
  if (threadIdx.x == 0) {
    T = classes;
    for (int s = 0; s < SW100_N_SITE_STATS; ++s) B.key[s] = 0u;
    B.nan_mask = B.nonfinite = B.codes = B.bad = 0u;
  }
  __syncthreads();
  PrepAcc A;
  for (int s = 0; s < SW100_N_SITE_STATS; ++s) A.key[s] = 0u;
  A.nan_mask = A.nonfinite = A.codes = A.bad = 0u;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x) {
    const float a = dsm[p], t2 = dem[p];
    float t1 = trees[p];
    if (t1 < 0.f) t1 = 0.f;                            // trees[trees < 0] = 0
    const float vegdem = t1 + t2;
    const float vegdem2 = t1 * 0.25f + t2;
    const float b = ((vegdem2 * vegdem == 0.f) ? 1.f : 0.f) * vegdem;  // logical_not(vegdem2 * vegdem) * vegdem
    float vd = t1 + a;
    if (vd == a) vd = 0.f;
    float vd2 = t1 * 0.25f + a;
    if (vd2 == a) vd2 = 0.f;
    const float h = a - t2;                            // buildings: < 2 -> 1, then >= 2 -> 0
    const float bld = (h < 2.f) ? 1.f : ((h >= 2.f) ? 0.f : h);
    vegdsm[p] = vd;
    vegdsm2[p] = vd2;
    if (bush) bush[p] = b;
    buildings[p] = bld;
    aspect_rad[p] = (aspect_deg[p] * 3.14159274101257324f) / 180.f;
    acc_max(A, SW100_STAT_DSM, a);
    acc_max(A, SW100_STAT_VEGDEM, vegdem);
    acc_max(A, SW100_STAT_VEGDSM, vd);
    acc_max(A, SW100_STAT_VEGDSM2, vd2);
    acc_max(A, SW100_STAT_ABS_DSM, fabsf(a));
    acc_max(A, SW100_STAT_ABS_VEGDSM, fabsf(vd));
    acc_max(A, SW100_STAT_ABS_VEGDSM2, fabsf(vd2));
    acc_max(A, SW100_STAT_BUSH, b);
    if (!isfinite(a) || !isfinite(vd) || !isfinite(vd2)) A.nonfinite = 1u;
    if (landcover) {
      float v = landcover[p];
      if (v < 1.f || v > 7.f) v = 6.f;                 // lc[(lc < 1) | (lc > 7)] = 6
      if (v == 3.f || v == 4.f) v = 5.f;               // lc[(lc == 3) | (lc == 4)] = 5
      const int code = (int)v;                         // 1..7 once the value is an integer
      if (v == (float)code && ((T.valid >> code) & 1u)) {
        tgk[p] = T.tgk[code];
        tstart[p] = T.tstart[code];
        alb[p] = T.alb[code];
        emis[p] = T.emis[code];
        class_idx[p] = (uint8_t)code;
        A.codes |= 1u << code;
      } else {                                         // no class row: the host refuses the site
        tgk[p] = tstart[p] = alb[p] = emis[p] = 0.f;
        class_idx[p] = 0;
        A.bad = 1u;
      }
    } else {                                           // zeros + the default class constants
      tgk[p] = 0.37f;
      tstart[p] = -3.41f;
      alb[p] = 0.15f;
      emis[p] = 0.95f;
      class_idx[p] = 0;
    }
  }
  // warp, block, grid
  for (int s = 0; s < SW100_N_SITE_STATS; ++s) A.key[s] = __reduce_max_sync(0xffffffffu, A.key[s]);
  A.nan_mask = __reduce_or_sync(0xffffffffu, A.nan_mask);
  A.nonfinite = __reduce_or_sync(0xffffffffu, A.nonfinite);
  A.codes = __reduce_or_sync(0xffffffffu, A.codes);
  A.bad = __reduce_or_sync(0xffffffffu, A.bad);
  if ((threadIdx.x & 31) == 0) {
    for (int s = 0; s < SW100_N_SITE_STATS; ++s) atomicMax(&B.key[s], A.key[s]);
    atomicOr(&B.nan_mask, A.nan_mask);
    atomicOr(&B.nonfinite, A.nonfinite);
    atomicOr(&B.codes, A.codes);
    atomicOr(&B.bad, A.bad);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < SW100_N_SITE_STATS; ++s) atomicMax(&stats->max_key[s], B.key[s]);
    atomicOr(&stats->nan_mask, B.nan_mask);
    atomicOr(&stats->nonfinite, B.nonfinite);
    atomicOr(&stats->codes, B.codes);
    atomicOr(&stats->bad_codes, B.bad);
  }
}

}  // namespace sw100
