// Wall-height sun march for every daytime step of a site in one launch.
//
// Reference: solweig_gpu/solweig.py:1079-1224 (shadowingfunction_wallheight_23)
// and the per-step shadow / ground-view-factor inputs of solweig.py:2094-2130
// and :75-128 (sunonsurface_2018a's Lup and sunwall planes).
//
// grid.z indexes the daytime step; one thread per pixel marches the step's
// table (index 0 = the self comparison, dzprev carried) and then writes the
// packed ground-view-factor source record {shadow, Lup, albedo, flags} that
// the time-loop kernel gathers 396 times per pixel and step.
#include "sw_common.cuh"
#include "sw_internal.cuh"

namespace sw100 {

struct MarchOut {
  float vegsh, sh, vbsh, wallsh, wallsun, wallshve, facesh, facesun;
};

// CHECKED false: the caller has shown that every step stays in the grid
// (the last step's cell is in it; the shifts grow monotonically in
// magnitude with one sign per axis).
template <bool CHECKED>
__device__ __forceinline__ MarchOut march_sun(const float4* __restrict__ src4, int rows, int cols, int r, int c,
                                              float a, float vegdem_p, float bush_p, float walls_p,
                                              float aspect_p, const sw100_step* __restrict__ steps, int n,
                                              float vmax, const sw100_sun_step& S) {
  // vegsh, sh and the "vbshvegsh ever counted" flag only take the values
  // 0 and 1 in the reference's float32 planes (vegsh starts at bushplant,
  // every update is a max with a 0/1 value or a reset to 0; vbshvegsh only
  // matters through > 0), so they are carried as booleans; f and shvoveg
  // stay float32 running maxima with torch.maximum's NaN rule.
  bool sh = false, vegsh = bush_p > 1.f, vb_any = false;
  float f = a;
  float shvoveg = vegdem_p;
  float dzprev = 0.f;
  const float wallbol = walls_p > 0.f ? 1.f : 0.f;
  const bool a_nonneg = nonneg(a);
  // Building shadow settles a pixel that is not a wall (walls exactly +0)
  // on finite rasters (vmax finite: no NaN or +inf source): from then on sh
  // stays 1, vegsh ends every step at 0 and vbsh gains nothing; f and
  // shvoveg only reach the outputs through the wall tail, where with walls
  // +0 they decide nothing but the sign of the zero (shvoveg - a) * 0,
  // which stays +0 once shvoveg - a is +0 or positive.
  const bool shade_exit = __float_as_uint(walls_p) == 0u && isfinite(vmax);
  for (int k = 0; k < n; ++k) {
    const sw100_step st = load_step(&steps[k]);
    const int sr = r + st.dx, sc = c + st.dy;
    const float dz = st.dz;
    float temp = 0.f, tv = 0.f, tv2 = 0.f, tlf = 0.f, tlg = 0.f;
    const bool inb = !CHECKED || in_grid(sr, sc, rows, cols);
    if (inb) {
      const float4 v = __ldg(&src4[(size_t)sr * cols + sc]);
      temp = __fsub_rn(v.x, dz);
      tv = __fsub_rn(v.y, dz);
      tv2 = __fsub_rn(v.z, dz);
      tlf = __fsub_rn(v.y, dzprev);
      tlg = __fsub_rn(v.z, dzprev);
    }
    f = tmax(f, temp);
    shvoveg = tmax(shvoveg, tv);
    sh = f > a;
    // vegsh2: 1 when one to three of the four canopy tests hold
    const int cnt = (int)(tv > a) + (int)(tv2 > a) + (int)(tlf > a) + (int)(tlg > a);
    dzprev = dz;
    vegsh = (vegsh || (cnt > 0 && cnt < 4)) && !sh;
    vb_any = vb_any || vegsh;
    // Nothing above this pixel can be reached any more: the ray has left the
    // grid (it stays out and reads zeros), or every later source height
    // minus a larger drop stays at or below the pixel, its running building
    // maximum and its running vegetation maximum.  Zeros are covered by
    // nonneg(a) and nonneg(shvoveg).
    const float top = __fsub_rn(vmax, dz);
    if (a_nonneg && nonneg(shvoveg) && (!inb || (top <= a && top <= shvoveg))) break;
    if (shade_exit && sh && nonneg(__fsub_rn(shvoveg, a))) break;
  }
  MarchOut o;
  float facesh;
  if (S.facesh_mode == 0) {
    facesh = ((aspect_p < S.facesh_lo || aspect_p >= S.facesh_hi) ? 1.f : 0.f) - wallbol + 1.f;
  } else {
    facesh = ((aspect_p > S.facesh_lo || aspect_p <= S.facesh_hi) ? 1.f : 0.f) * -1.f + 1.f;
  }
  const float vegf = vegsh ? 1.f : 0.f;
  const float shf = 1.f - (sh ? 1.f : 0.f);
  float vbsh = (vb_any ? 1.f : 0.f) - vegf;
  shvoveg = (shvoveg - a) * vegf;
  const float vegshf = 1.f - vegf;
  vbsh = 1.f - vbsh;
  const float shvo = f - a;
  const float facesun = ((facesh + wallbol == 1.f) && walls_p > 0.f) ? 1.f : 0.f;
  float wallsun = walls_p - shvo;
  if (wallsun < 0.f) wallsun = 0.f;
  if (facesh == 1.f) wallsun = 0.f;
  const float wallsh = walls_p - wallsun;
  float wallshve = shvoveg * wallbol;
  wallshve = wallshve - wallsh;
  if (wallshve < 0.f) wallshve = 0.f;
  wallsun = wallsun - wallshve;
  if (wallsun < 0.f) wallsun = 0.f;
  if (wallshve > walls_p) wallshve = walls_p;
  o.vegsh = vegshf; o.sh = shf; o.vbsh = vbsh; o.wallsh = wallsh; o.wallsun = wallsun;
  o.wallshve = wallshve; o.facesh = facesh; o.facesun = facesun;
  return o;
}

// Daytime row d of pixel (r, c): march, wall tail and the ground-view-factor
// source record.  `Site` is SitePlanes or sw100_site_planes.
template <class Site>
__device__ __forceinline__ void sun_march_pixel(const float4* __restrict__ src4, const Site& site, int rows, int cols,
                                                const sw100_sun_step* __restrict__ sun_steps,
                                                const sw100_time_step* __restrict__ tsteps,
                                                const sw100_step* __restrict__ table, float vmax,
                                                float4* __restrict__ gsrc, float* __restrict__ debug8, int r, int c,
                                                int d) {
  const size_t npix = (size_t)rows * cols;
  const size_t p = (size_t)r * cols + c;
  const sw100_sun_step S = sun_steps[d];
  const float4 self = src4[p];
  const float walls_p = site.walls[p];
  const sw100_step* steps = table + S.step_offset;
  // a march whose last cell is in the grid never leaves it
  bool inside = false;
  if (S.step_count > 0) {
    const sw100_step last = load_step(&steps[S.step_count - 1]);
    inside = in_grid(r + last.dx, c + last.dy, rows, cols);
  }
  const MarchOut o = inside
      ? march_sun<false>(src4, rows, cols, r, c, self.x, self.y, self.w, walls_p, site.aspect_rad[p], steps,
                         S.step_count, vmax, S)
      : march_sun<true>(src4, rows, cols, r, c, self.x, self.y, self.w, walls_p, site.aspect_rad[p], steps,
                        S.step_count, vmax, S);
  const float shadow = o.sh - (1.f - o.vegsh) * S.psi_term;
  // sunonsurface_2018a inputs at this pixel (solweig.py:118-128, gvf_2018a :342)
  const sw100_time_step& P = tsteps[S.t];
  const float bld = site.buildings[p];
  const float tg = ground_temperature(site, P, p);
  const float sbc_emis = P.sbc * site.emis[p];
  const float lup = sbc_emis * pow4f(tg * shadow + P.ta32 + 273.15f) - sbc_emis * P.ta4;
  const float sunwall = ((o.wallsun / walls_p) * bld == 1.f) ? 1.f : 0.f;
  const uint32_t flags = (bld != 0.f ? 1u : 0u) | (sunwall != 0.f ? 2u : 0u) | (bld == 1.f ? 4u : 0u);
  gsrc[d * npix + p] = make_float4(shadow, lup, site.alb[p], __uint_as_float(flags));
  if (debug8) {
    float* o8 = debug8 + (size_t)d * 8 * npix + p;
    o8[0 * npix] = o.vegsh; o8[1 * npix] = o.sh; o8[2 * npix] = o.vbsh; o8[3 * npix] = o.wallsh;
    o8[4 * npix] = o.wallsun; o8[5 * npix] = o.wallshve; o8[6 * npix] = o.facesh; o8[7 * npix] = o.facesun;
  }
}

__global__ void __launch_bounds__(256) sun_march_kernel(const float4* __restrict__ src4, SitePlanes site, int rows,
                                                         int cols, const sw100_sun_step* __restrict__ sun_steps,
                                                         const sw100_time_step* __restrict__ tsteps,
                                                         const sw100_step* __restrict__ table, float vmax,
                                                         float4* __restrict__ gsrc, float* __restrict__ debug8) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  if (r >= rows || c >= cols) return;
  sun_march_pixel(src4, site, rows, cols, sun_steps, tsteps, table, vmax, gsrc, debug8, r, c, blockIdx.z);
}

// Sun march of every daytime row of every site of a batch: each tile
// carries its daytime row.
__global__ void __launch_bounds__(128) sun_march_batch_kernel(const sw100_batch_site* __restrict__ sites,
                                                              const sw100_tile* __restrict__ tiles, int n_tiles) {
  for (int i = blockIdx.x; i < n_tiles; i += gridDim.x) {
    const sw100_tile T = tiles[i];
    const sw100_batch_site& S = sites[T.site];
    const int c = T.tx * blockDim.x + threadIdx.x;
    const int r = T.ty * blockDim.y + threadIdx.y;
    if (r >= S.rows || c >= S.cols || T.day >= S.series.n_day) continue;
    sun_march_pixel(reinterpret_cast<const float4*>(S.src4), S.site, S.rows, S.cols, S.series.sun, S.series.steps,
                    S.series.sun_table, S.site.vmax, reinterpret_cast<float4*>(S.gsrc), nullptr, r, c, T.day);
  }
}

}  // namespace sw100
