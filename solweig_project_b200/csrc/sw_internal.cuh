// Internal kernel-side structures shared by the time-loop kernels.
#pragma once

#include "sw_common.cuh"

namespace sw100 {

// Device view of sw100_site_planes (passed by value as a kernel argument).
struct SitePlanes {
  const float* svfbuveg;
  const float* hsvf;
  const float* tan_alfa;
  const float* buildings;
  const float* walls;
  const float* aspect_rad;
  const float* tgk;
  const float* tstart;
  const float* alb;
  const float* emis;
  const uint8_t* class_idx;
  const float* windcoeff;
  const uint32_t* bits;
  uint32_t single_step[SW100_CUBE_WORDS];
  const int32_t* patch_order;
  int32_t n_patch_order;
};

__host__ inline SitePlanes make_site(const sw100_site_planes& s) {
  SitePlanes d;
  d.svfbuveg = s.svfbuveg; d.hsvf = s.hsvf; d.tan_alfa = s.tan_alfa; d.buildings = s.buildings;
  d.walls = s.walls; d.aspect_rad = s.aspect_rad; d.tgk = s.tgk; d.tstart = s.tstart; d.alb = s.alb;
  d.emis = s.emis; d.class_idx = s.class_idx; d.windcoeff = s.windcoeff; d.bits = s.bits;
  for (int w = 0; w < SW100_CUBE_WORDS; ++w) d.single_step[w] = s.single_step[w];
  d.patch_order = s.patch_order;
  d.n_patch_order = s.n_patch_order;
  return d;
}

// Ground temperature of the daytime parameterisation (solweig.py:2102-2122):
// Tg = (TgK * altmax + Tstart) * sin-wave factor of the pixel's TmaxLST class,
// times CI_TgG, floored at 0 when land cover is used.
// (`Site` is SitePlanes or sw100_site_planes: the same member names.)
template <class Site>
__device__ __forceinline__ float ground_temperature(const Site& site, const sw100_time_step& P, size_t p) {
  const float tgamp = site.tgk[p] * P.altmax32 + site.tstart[p];
  float tg = tgamp * P.tg_factor[min((int)site.class_idx[p], SW100_MAX_CLASSES - 1)];
  tg = tg * P.cig;
  if (P.landcover) tg = tmax(tg, 0.f);
  return tg;
}

}  // namespace sw100
