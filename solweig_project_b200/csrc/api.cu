// C ABI of the library (see include/solweig_b200.h for the contract).
//
// Mirrors the reference's native ABI conventions (native/cuda/src/sw_api.cu:
// extern "C", status return, last-error string per thread) but never
// allocates: every scratch buffer comes from the caller's workspace, so the
// entry points can be captured in CUDA graphs and driven from any allocator.
#include <algorithm>
#include <cmath>
#include <climits>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include <cuda_bf16.h>

#include "sw_common.cuh"
#include "sw_internal.cuh"

namespace sw100 {
__global__ void pack4_kernel(const float* a, const float* b, const float* c, const float* d, size_t n, float4* out);
__global__ void svf_sweep_kernel(const float4* src4, int rows, int cols, const sw100_svf_plan* plan_g,
                                 const sw100_step* steps, const uint32_t* bflags, float vmax, float* out,
                                 uint32_t* bits, int n_steps, const float* skipmap, unsigned int* next, int n_patch);
__global__ void svf_sweep_count_kernel(const float4* src4, int rows, int cols, const sw100_svf_plan* plan_g,
                                       const sw100_step* steps, const uint32_t* bflags, float vmax, float* out,
                                       uint32_t* bits, int n_steps, const float* skipmap,
                                       unsigned long long* executed);
__global__ void svf_skipmap_kernel(const float4* src4, int rows, int cols, float* m, int crow, int ccol);
__global__ void svf_statics_kernel(float* planes, int64_t npix, float trans_veg);
__global__ void svf_window_kernel(const float4* src4, int rows, int cols, const sw100_svf_plan* plan_g,
                                  const sw100_step* steps, const int32_t* corridor, float vmax, int4 rect, int4 win,
                                  float* out, uint32_t* bits, int n_steps);
__global__ void svf_box_pairs_kernel(const float4* src4, int rows, int cols, const sw100_svf_plan* plan,
                                     const sw100_step* steps, float vmax, int4 box, uint32_t* bits, int n_steps);
__global__ void diff_bbox_kernel(const float4* a, const float4* b, int rows, int cols, int* box);
__global__ void box_init_kernel(int* box);
__global__ void pack_batch_kernel(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles);
__global__ void svf_bush_flags_batch_kernel(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles);
__global__ void svf_sweep_batch_kernel(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles);
__global__ void sun_march_batch_kernel(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles);
__global__ void skipmap_batch_kernel(const sw100_batch_site* sites);
__global__ void time_loop_batch_kernel(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles);
__global__ void time_loop_batch_sums_kernel(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles);
__global__ void svf_bush_flags_kernel(const float4* src4, int rows, int cols, const sw100_svf_plan* plan,
                                      const sw100_step* steps, uint32_t* flags, int n_steps);
__global__ void sun_march_kernel(const float4* src4, SitePlanes site, int rows, int cols,
                                 const sw100_sun_step* sun_steps, const sw100_time_step* tsteps,
                                 const sw100_step* table, float vmax, float4* gsrc, float* debug8);
__global__ void time_loop_kernel(SitePlanes site, int rows, int cols, const sw100_time_step* tsteps, int n_t,
                                 const sw100_patch_step* patch_steps, int n_patches,
                                 const sw100_gvf_azimuth* gvf_az, const float4* gsrc, int n_day, float* state,
                                 uint32_t out_mask, float* outputs);
__global__ void time_loop_sums_kernel(SitePlanes site, int rows, int cols, const sw100_time_step* tsteps, int n_t,
                                      const sw100_patch_step* patch_steps, int n_patches,
                                      const sw100_gvf_azimuth* gvf_az, const float4* gsrc, int n_day, float* state,
                                      uint32_t out_mask, float* outputs, const float* sums);
__global__ void walk_work_kernel(const float* buildings, int rows, int cols, const sw100_gvf_azimuth* gvf, int second,
                                 int32_t* work, int n_patch);
__global__ void patch_weights_kernel(const sw100_time_step* steps, int n_t, const sw100_patch_step* patch,
                                     int n_patches, __nv_bfloat16* W, int n_groups);
__global__ void patch_sums_tc_kernel(const uint32_t* bits, int64_t npix, int n_patches, const __nv_bfloat16* W,
                                     int n_groups, int n_t, float* sums, int* err, int wait_limit);
__global__ void pack_cubes_kernel(const float* sh, const float* veg, const float* vb, size_t npix, int n_patches,
                                  Single5 single, uint32_t* bits);
__global__ void utci_steps_kernel(const sw100_time_step* steps, int n_steps, const float* tmrt,
                                  const float* buildings, const float* windcoeff, int64_t npix, float* out);
__global__ void utci_kernel(const float* ta, const float* rh, const float* tmrt, const float* va, int64_t n,
                            float* out);
__global__ void nn_conv3x3_tc_kernel(const __nv_bfloat16* X, int N, int H, int W, int Cin, int xstride, int xcoff,
                                     const __nv_bfloat16* Wt, const float* bias, int Cout, void* Yv, int ystride,
                                     int ycoff, int relu, int out_f32, int* err, int wait_limit);
__global__ void nn_wgrad_kernel(const __nv_bfloat16* X, int N, int H, int W, int Cin, int xstride, int xcoff,
                                const __nv_bfloat16* dY, int Cout, int dstride, int dcoff, float* dW, float* dbias,
                                int rows_per_block);
__global__ void prepare_site_kernel(const float* dsm, const float* trees, const float* dem, const float* aspect_deg,
                                    const float* landcover, sw100_class_table classes, size_t npix, float* vegdsm,
                                    float* vegdsm2, float* bush, float* buildings, float* aspect_rad, float* tgk,
                                    float* tstart, float* alb, float* emis, uint8_t* class_idx,
                                    sw100_site_stats* stats);
__global__ void nn_weights_kernel(const float* Wm, int Cin, int Cout, __nv_bfloat16* Wf, __nv_bfloat16* Wd);
__global__ void nn_relu_bwd_kernel(__nv_bfloat16* dY, const __nv_bfloat16* Y, int64_t npix, int C, int dstride,
                                   int dcoff, int ystride, int ycoff);
__global__ void nn_pool2_kernel(const __nv_bfloat16* X, int N, int H, int W, int C, int xstride, int xcoff,
                                __nv_bfloat16* Y, int ystride, int ycoff);
__global__ void nn_pool2_bwd_kernel(const __nv_bfloat16* dY, int N, int H, int W, int C, int dstride, int dcoff,
                                    __nv_bfloat16* dX, int xstride, int xcoff, int accumulate);
__global__ void nn_up2_kernel(const __nv_bfloat16* X, int N, int H, int W, int C, int xstride, int xcoff,
                              __nv_bfloat16* Y, int ystride, int ycoff);
__global__ void nn_up2_bwd_kernel(const __nv_bfloat16* dY, int N, int H, int W, int C, int dstride, int dcoff,
                                  __nv_bfloat16* dX, int xstride, int xcoff);
__global__ void nn_mse_kernel(const float* pred, const float* target, int N, int H, int W, int C, int nc, int m,
                              float inv_count, __nv_bfloat16* dpred, float* loss);
__global__ void nn_adam_kernel(float* p, const float* grad, float* m, float* v, int64_t n, float lr, float b1,
                               float b2, float eps, float c1, float c2);
__global__ void nn_input_kernel(const float* dsm, const float* vegdsm, const float* vegdsm2, const float* dem,
                                int rows, int cols, const int2* origins, int n, int S, __nv_bfloat16* X);
}  // namespace sw100

using namespace sw100;

namespace {

thread_local std::string g_last_error;
std::atomic<int64_t> g_launches{0};
// polls of an mbarrier before a tensor-core kernel's wait gives up
constexpr int kDefaultTcWaitLimit = 1 << 22;
std::atomic<int> g_tc_wait_limit{kDefaultTcWaitLimit};

constexpr int64_t kMaxPixels = int64_t(1) << 31;  // int32 pixel offsets inside kernels
constexpr int64_t kAlign = 256;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail((int)e, "%s: %s", what, cudaGetErrorString(e));
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return 0;
}

int64_t align_up(int64_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Block shape of the march kernels (SVF sweep, windowed recompute): 128
// threads, a warp covering 8 x 4 pixels.
constexpr int kMarchBx = 8, kMarchBy = 16;
// Block shape of the time / flux loops: 128 threads, a warp covering 8 x 4
// pixels.  A warp's ground-view walks last as long as its longest one, and
// the first-building step varies less over an 8 x 4 patch than along a row
// of 32 (a quarter fewer walk steps per warp at 500 x 500, 8 % faster loop).
constexpr int kLoopBx = 8, kLoopBy = 16;
constexpr int kTimeLoopThreads = 128;  // threads of a time-loop block (kTileThreads of time_loop.cu)

int check_grid(int rows, int cols) {
  if (rows <= 0 || cols <= 0) return fail(SW100_E_SIZE, "grid %d x %d must be positive", rows, cols);
  if ((int64_t)rows * cols >= kMaxPixels) return fail(SW100_E_SIZE, "grid %d x %d too large", rows, cols);
  return 0;
}

int check_ptr(const void* p, const char* name) {
  if (!p) return fail(SW100_E_ARG, "%s must not be NULL", name);
  return 0;
}

int check_workspace(const void* ws, int64_t have, int64_t need) {
  if (need > 0 && (!ws || have < need))
    return fail(SW100_E_WORKSPACE, "workspace of %lld bytes required, %lld given", (long long)need,
                (long long)(ws ? have : 0));
  if (ws && (reinterpret_cast<uintptr_t>(ws) % 16) != 0) return fail(SW100_E_ARG, "workspace must be 16-byte aligned");
  return 0;
}

int launch_pack(const sw100_site_planes& s, int rows, int cols, float4* out, cudaStream_t st) {
  const size_t n = (size_t)rows * cols;
  const int threads = 256;
  const int blocks = (int)std::min<size_t>((n + threads - 1) / threads, 148 * 16);
  pack4_kernel<<<blocks, threads, 0, st>>>(s.dsm, s.vegdsm, s.vegdsm2, s.bush_any ? s.bush : nullptr, n, out);
  return check_launch("pack4_kernel");
}

int validate_site_march(const sw100_site_planes* s) {
  int rc;
  if ((rc = check_ptr(s, "site"))) return rc;
  if ((rc = check_ptr(s->dsm, "site->dsm"))) return rc;
  if ((rc = check_ptr(s->vegdsm, "site->vegdsm"))) return rc;
  if ((rc = check_ptr(s->vegdsm2, "site->vegdsm2"))) return rc;
  if (s->bush_any && !s->bush) return fail(SW100_E_ARG, "site->bush is NULL but bush_any is set");
  return 0;
}

int validate_site_loop(const sw100_site_planes* s) {
  int rc;
  if ((rc = validate_site_march(s))) return rc;
  const void* ptrs[] = {s->svfbuveg, s->hsvf, s->tan_alfa, s->buildings, s->walls, s->aspect_rad, s->tgk,
                        s->tstart, s->alb, s->emis, s->class_idx, s->windcoeff, s->bits};
  const char* names[] = {"svfbuveg", "hsvf", "tan_alfa", "buildings", "walls", "aspect_rad", "tgk",
                         "tstart", "alb", "emis", "class_idx", "windcoeff", "bits"};
  for (int i = 0; i < 13; ++i)
    if (!ptrs[i]) return fail(SW100_E_ARG, "site->%s must not be NULL", names[i]);
  return 0;
}

int validate_series(const sw100_series* s) {
  int rc;
  if ((rc = check_ptr(s, "series"))) return rc;
  if (s->n_t <= 0) return fail(SW100_E_ARG, "series->n_t must be positive");
  if (s->n_day < 0 || s->n_day > s->n_t) return fail(SW100_E_ARG, "series->n_day out of range");
  if (s->n_day > 65535) return fail(SW100_E_SIZE, "too many daytime steps");
  if (s->n_patches <= 0 || s->n_patches > 153) return fail(SW100_E_SIZE, "series->n_patches must be 1..153");
  if ((rc = check_ptr(s->steps, "series->steps"))) return rc;
  if ((rc = check_ptr(s->patch, "series->patch"))) return rc;
  if ((rc = check_ptr(s->gvf, "series->gvf"))) return rc;
  if (s->n_day > 0) {
    if ((rc = check_ptr(s->sun, "series->sun"))) return rc;
    if ((rc = check_ptr(s->sun_table, "series->sun_table"))) return rc;
  }
  return 0;
}

// Bytes of a site's skip map (one float per 8 x 8 cell block), aligned.
// Blocks of `threads` threads of `kernel` resident on the current device at
// once (occupancy x SM count): the grid of a persistent kernel.
template <class K>
int resident_blocks(K kernel, int threads, int* blocks) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  if (e != cudaSuccess) return fail((int)e, "occupancy query: %s", cudaGetErrorString(e));
  *blocks = std::max(1, per_sm) * std::max(1, sms);
  return 0;
}

int64_t skipmap_bytes(int rows, int cols) { return align_up((int64_t)((rows + 7) / 8) * ((cols + 7) / 8) * 4); }

int launch_skipmap(const float4* src4, int rows, int cols, float* skipmap, cudaStream_t st) {
  const int crow = (rows + 7) / 8, ccol = (cols + 7) / 8;
  const long long threads = (long long)crow * ccol * 32;  // one warp per 8 x 8 block
  svf_skipmap_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(src4, rows, cols, skipmap, crow, ccol);
  return check_launch("svf_skipmap_kernel");
}

int launch_sun_march(const sw100_site_planes& site, int rows, int cols, const sw100_series& ser, const float4* src4,
                     float4* gsrc, float* debug8, cudaStream_t st) {
  if (ser.n_day == 0) return 0;
  // 8 x 32 blocks: warps of 8 x 4 pixels (see the sweep)
  const dim3 block(8, 32);
  const dim3 grid((cols + 7) / 8, (rows + 31) / 32, ser.n_day);
  sun_march_kernel<<<grid, block, 0, st>>>(src4, make_site(site), rows, cols, ser.sun, ser.steps, ser.sun_table,
                                           site.vmax, gsrc, debug8);
  return check_launch("sun_march_kernel");
}

// Launch shape of the time / flux loops: four 8 x 4 pixel patches per block
// in the site's patch order, or 8 x 16 blocks in grid order without one.
int loop_shape(const sw100_site_planes& site, int rows, int cols, dim3& grid, dim3& block) {
  if (site.patch_order == nullptr) {
    block = dim3(kLoopBx, kLoopBy);
    grid = dim3((cols + kLoopBx - 1) / kLoopBx, (rows + kLoopBy - 1) / kLoopBy);
    return 0;
  }
  const int64_t n = (int64_t)((rows + 3) / 4) * ((cols + 7) / 8);
  if (site.n_patch_order != n)
    return fail(SW100_E_ARG, "n_patch_order %d must be %lld (8 x 4 patches of a %d x %d grid)", site.n_patch_order,
                (long long)n, rows, cols);
  block = dim3(kTimeLoopThreads);
  grid = dim3((unsigned)((n + 3) / 4));
  return 0;
}

}  // namespace

extern "C" {

int sw100_abi_version(void) { return SW100_ABI_VERSION; }

const char* sw100_last_error(void) { return g_last_error.c_str(); }

int64_t sw100_launch_count(void) { return g_launches.load(); }

int sw100_svf_workspace_bytes(int rows, int cols, int n_steps, int64_t* bytes) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = check_ptr(bytes, "bytes"))) return rc;
  if (n_steps < 0) return fail(SW100_E_ARG, "n_steps must be >= 0");
  // packed rasters, bush flags, skip map, the persistent sweep's patch counter
  *bytes = align_up((int64_t)rows * cols * 16) + align_up((int64_t)n_steps * 4) + skipmap_bytes(rows, cols) +
           kAlign;
  return 0;
}

}  // extern "C"

namespace {
// Packing, bush flags and skip map of a sweep, then the sweep itself (the
// counting kernel when `executed` is set).
int run_svf_sweep(const sw100_site_planes* site, int rows, int cols, const sw100_svf_plan* plan,
                  const sw100_step* steps, int n_steps, float* out_planes, uint32_t* out_bits, void* workspace,
                  int64_t workspace_bytes, unsigned long long* executed, void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = validate_site_march(site))) return rc;
  if ((rc = check_ptr(plan, "plan")) || (rc = check_ptr(steps, "steps")) || (rc = check_ptr(out_planes, "out_planes")) ||
      (rc = check_ptr(out_bits, "out_bits")))
    return rc;
  int64_t need = 0;
  if ((rc = sw100_svf_workspace_bytes(rows, cols, n_steps, &need))) return rc;
  if ((rc = check_workspace(workspace, workspace_bytes, need))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float4* src4 = static_cast<float4*>(workspace);
  uint32_t* flags = reinterpret_cast<uint32_t*>(static_cast<char*>(workspace) + align_up((int64_t)rows * cols * 16));
  if ((rc = launch_pack(*site, rows, cols, src4, st))) return rc;
  dim3 block(32, 4);
  dim3 grid((cols + 31) / 32, (rows + 3) / 4);
  if (site->bush_any) {
    cudaError_t e = cudaMemsetAsync(flags, 0, (size_t)n_steps * 4, st);
    if (e != cudaSuccess) return fail((int)e, "cudaMemsetAsync: %s", cudaGetErrorString(e));
    svf_bush_flags_kernel<<<grid, block, 0, st>>>(src4, rows, cols, plan, steps, flags, n_steps);
    if ((rc = check_launch("svf_bush_flags_kernel"))) return rc;
  }
  // skip map after the bush flags
  float* skipmap = reinterpret_cast<float*>(reinterpret_cast<char*>(flags) + align_up((int64_t)n_steps * 4));
  if ((rc = launch_skipmap(src4, rows, cols, skipmap, st))) return rc;
  // 8 x 16 blocks: a warp marches an 8 x 4 pixel patch, whose rays meet
  // similar obstacles (less divergence than a 32 x 1 row: -20 % time)
  const dim3 sblock(kMarchBx, kMarchBy);
  const dim3 sgrid((cols + kMarchBx - 1) / kMarchBx, (rows + kMarchBy - 1) / kMarchBy);
  if (executed == nullptr) {
    unsigned int* next = reinterpret_cast<unsigned int*>(reinterpret_cast<char*>(skipmap) + skipmap_bytes(rows, cols));
    cudaError_t e = cudaMemsetAsync(next, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return fail((int)e, "cudaMemsetAsync: %s", cudaGetErrorString(e));
    const int n_patch = ((rows + 3) / 4) * ((cols + 7) / 8);
    int blocks = 0;
    if ((rc = resident_blocks(svf_sweep_kernel, 128, &blocks))) return rc;
    blocks = std::max(1, std::min(blocks, (n_patch + 3) / 4));
    svf_sweep_kernel<<<blocks, 128, 0, st>>>(src4, rows, cols, plan, steps, site->bush_any ? flags : nullptr,
                                             site->vmax, out_planes, out_bits, n_steps, skipmap, next, n_patch);
    return check_launch("svf_sweep_kernel");
  }
  cudaError_t e = cudaMemsetAsync(executed, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return fail((int)e, "cudaMemsetAsync: %s", cudaGetErrorString(e));
  svf_sweep_count_kernel<<<sgrid, sblock, 0, st>>>(src4, rows, cols, plan, steps, site->bush_any ? flags : nullptr,
                                                   site->vmax, out_planes, out_bits, n_steps, skipmap, executed);
  return check_launch("svf_sweep_count_kernel");
}
}  // namespace

extern "C" {

int sw100_svf_sweep(const sw100_site_planes* site, int rows, int cols, const sw100_svf_plan* plan,
                    const sw100_step* steps, int n_steps, float* out_planes, uint32_t* out_bits, void* workspace,
                    int64_t workspace_bytes, void* stream) {
  return run_svf_sweep(site, rows, cols, plan, steps, n_steps, out_planes, out_bits, workspace, workspace_bytes,
                       nullptr, stream);
}

int sw100_svf_statics(float* planes, int rows, int cols, float trans_veg, void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = check_ptr(planes, "planes"))) return rc;
  const int64_t npix = (int64_t)rows * cols;
  const int blocks = (int)std::min<int64_t>((npix + 255) / 256, 148 * 8);
  svf_statics_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(planes, npix, trans_veg);
  return check_launch("svf_statics_kernel");
}

int sw100_svf_sweep_count(const sw100_site_planes* site, int rows, int cols, const sw100_svf_plan* plan,
                          const sw100_step* steps, int n_steps, float* out_planes, uint32_t* out_bits,
                          void* workspace, int64_t workspace_bytes, uint64_t* executed, void* stream) {
  int rc;
  if ((rc = check_ptr(executed, "executed"))) return rc;
  return run_svf_sweep(site, rows, cols, plan, steps, n_steps, out_planes, out_bits, workspace, workspace_bytes,
                       reinterpret_cast<unsigned long long*>(executed), stream);
}

int sw100_svf_window_workspace_bytes(int rows, int cols, int64_t* bytes) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = check_ptr(bytes, "bytes"))) return rc;
  *bytes = align_up((int64_t)rows * cols * 16);
  return 0;
}

int sw100_svf_window(const sw100_site_planes* site, int rows, int cols, const sw100_svf_plan* plan,
                     const sw100_step* steps, int n_steps, const int32_t* corridor, const int32_t rect[4],
                     const int32_t window[4], float* planes, uint32_t* bits, void* workspace,
                     int64_t workspace_bytes, void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = validate_site_march(site))) return rc;
  if ((rc = check_ptr(plan, "plan")) || (rc = check_ptr(steps, "steps")) || (rc = check_ptr(corridor, "corridor")) ||
      (rc = check_ptr(rect, "rect")) || (rc = check_ptr(window, "window")) || (rc = check_ptr(planes, "planes")) ||
      (rc = check_ptr(bits, "bits")))
    return rc;
  if (site->bush_any) return fail(SW100_E_ARG, "windowed recompute refuses rasters with bush");
  if (n_steps < 0) return fail(SW100_E_ARG, "n_steps must be >= 0");
  const int w0 = window[0], w1 = window[1], w2 = window[2], w3 = window[3];
  if (w0 < 0 || w1 >= rows || w2 < 0 || w3 >= cols || w0 > w1 || w2 > w3)
    return fail(SW100_E_ARG, "window {%d, %d, %d, %d} must be a non-empty box inside the %d x %d grid", w0, w1, w2,
                w3, rows, cols);
  if (rect[0] > rect[1] || rect[2] > rect[3]) return fail(SW100_E_ARG, "rect must be non-empty");
  int64_t need = 0;
  if ((rc = sw100_svf_window_workspace_bytes(rows, cols, &need))) return rc;
  if ((rc = check_workspace(workspace, workspace_bytes, need))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float4* src4 = static_cast<float4*>(workspace);
  if ((rc = launch_pack(*site, rows, cols, src4, st))) return rc;
  const dim3 block(kMarchBx, kMarchBy);
  const dim3 grid((w3 - w2 + 1 + kMarchBx - 1) / kMarchBx, (w1 - w0 + 1 + kMarchBy - 1) / kMarchBy);
  svf_window_kernel<<<grid, block, 0, st>>>(src4, rows, cols, plan, steps, corridor, site->vmax,
                                            make_int4(rect[0], rect[1], rect[2], rect[3]),
                                            make_int4(w0, w1, w2, w3), planes, bits, n_steps);
  return check_launch("svf_window_kernel");
}

int sw100_svf_box(const sw100_site_planes* site, int rows, int cols, const sw100_svf_plan* plan,
                  const sw100_step* steps, int n_steps, const int32_t* corridor, const int32_t box[4], float* planes,
                  uint32_t* bits, void* workspace, int64_t workspace_bytes, void* stream) {
  int rc;
  if (n_steps < 0) return fail(SW100_E_ARG, "n_steps must be >= 0");
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = validate_site_march(site))) return rc;
  if ((rc = check_ptr(plan, "plan")) || (rc = check_ptr(steps, "steps")) || (rc = check_ptr(corridor, "corridor")) ||
      (rc = check_ptr(box, "box")) || (rc = check_ptr(planes, "planes")) || (rc = check_ptr(bits, "bits")))
    return rc;
  if (site->bush_any) return fail(SW100_E_ARG, "box recompute refuses rasters with bush");
  if (box[0] < 0 || box[1] >= rows || box[2] < 0 || box[3] >= cols || box[0] > box[1] || box[2] > box[3])
    return fail(SW100_E_ARG, "box must be a non-empty box inside the grid");
  int64_t need = 0;
  if ((rc = sw100_svf_window_workspace_bytes(rows, cols, &need))) return rc;
  if ((rc = check_workspace(workspace, workspace_bytes, need))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float4* src4 = static_cast<float4*>(workspace);
  if ((rc = launch_pack(*site, rows, cols, src4, st))) return rc;
  const int4 b4 = make_int4(box[0], box[1], box[2], box[3]);
  const int64_t pairs = (int64_t)(box[1] - box[0] + 1) * (box[3] - box[2] + 1) * SW100_MAX_PATCHES;
  const int blocks = (int)std::min<int64_t>((pairs + 127) / 128, 148 * 32);
  svf_box_pairs_kernel<<<blocks, 128, 0, st>>>(src4, rows, cols, plan, steps, site->vmax, b4, bits, n_steps);
  if ((rc = check_launch("svf_box_pairs_kernel"))) return rc;
  // re-accumulate from the new bits: a rectangle outside the grid, read by no march
  const dim3 block(kMarchBx, kMarchBy);
  const dim3 grid((box[3] - box[2] + 1 + kMarchBx - 1) / kMarchBx, (box[1] - box[0] + 1 + kMarchBy - 1) / kMarchBy);
  svf_window_kernel<<<grid, block, 0, st>>>(src4, rows, cols, plan, steps, corridor, site->vmax,
                                            make_int4(-4, -4, -4, -4), b4, planes, bits, n_steps);
  return check_launch("svf_window_kernel");
}

int sw100_diff_bbox_workspace_bytes(int rows, int cols, int64_t* bytes) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = check_ptr(bytes, "bytes"))) return rc;
  *bytes = 2 * align_up((int64_t)rows * cols * 16);
  return 0;
}

int sw100_diff_bbox(const sw100_site_planes* before, const sw100_site_planes* after, int rows, int cols,
                    int32_t* box, void* workspace, int64_t workspace_bytes, void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = validate_site_march(before)) || (rc = validate_site_march(after))) return rc;
  if ((rc = check_ptr(box, "box"))) return rc;
  int64_t need = 0;
  if ((rc = sw100_diff_bbox_workspace_bytes(rows, cols, &need))) return rc;
  if ((rc = check_workspace(workspace, workspace_bytes, need))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float4* a = static_cast<float4*>(workspace);
  float4* b = reinterpret_cast<float4*>(static_cast<char*>(workspace) + align_up((int64_t)rows * cols * 16));
  if ((rc = launch_pack(*before, rows, cols, a, st))) return rc;
  if ((rc = launch_pack(*after, rows, cols, b, st))) return rc;
  box_init_kernel<<<1, 32, 0, st>>>(box);
  if ((rc = check_launch("box_init_kernel"))) return rc;
  const size_t n = (size_t)rows * cols;
  const int threads = 256;
  const int blocks = (int)std::min<size_t>((n + threads - 1) / threads, 148 * 8);
  diff_bbox_kernel<<<blocks, threads, 0, st>>>(a, b, rows, cols, box);
  return check_launch("diff_bbox_kernel");
}

int sw100_batch_validate(const sw100_batch_site* host_sites, int n_sites) {
  int rc;
  if (n_sites < 0) return fail(SW100_E_ARG, "n_sites must be >= 0");
  if (n_sites > 0 && (rc = check_ptr(host_sites, "host_sites"))) return rc;
  for (int i = 0; i < n_sites; ++i) {
    const sw100_batch_site& b = host_sites[i];
    if ((rc = check_grid(b.rows, b.cols))) return fail(rc, "site %d: %s", i, g_last_error.c_str());
    if ((rc = validate_site_march(&b.site))) return fail(rc, "site %d: %s", i, g_last_error.c_str());
    const void* ptrs[] = {b.plan, b.steps, b.svf_planes, b.svf_bits, b.src4, b.state};
    const char* names[] = {"plan", "steps", "svf_planes", "svf_bits", "src4", "state"};
    for (int k = 0; k < 6; ++k)
      if (!ptrs[k]) return fail(SW100_E_ARG, "site %d: %s must not be NULL", i, names[k]);
    if (b.site.bush_any && !b.bflags) return fail(SW100_E_ARG, "site %d: bflags must not be NULL with bush", i);
    if (b.svf_steps < 0) return fail(SW100_E_ARG, "site %d: svf_steps must be >= 0", i);
    if ((rc = validate_series(&b.series))) return fail(rc, "site %d: %s", i, g_last_error.c_str());
    if (b.series.n_day > 0 && !b.gsrc) return fail(SW100_E_ARG, "site %d: gsrc must not be NULL", i);
    if (b.out_mask & ~0x7Fu) return fail(SW100_E_ARG, "site %d: unknown output bits 0x%x", i, b.out_mask);
    if (b.out_mask && !b.outputs) return fail(SW100_E_ARG, "site %d: outputs must not be NULL", i);
    if (b.site.bits != b.svf_bits || b.site.svfbuveg != b.svf_planes + (size_t)16 * b.rows * b.cols ||
        b.site.hsvf != b.svf_planes + (size_t)17 * b.rows * b.cols ||
        b.site.tan_alfa != b.svf_planes + (size_t)18 * b.rows * b.cols)
      return fail(SW100_E_ARG, "site %d: site statics must point into svf_planes / svf_bits", i);
    const void* loop[] = {b.site.buildings, b.site.walls, b.site.aspect_rad, b.site.tgk, b.site.tstart,
                          b.site.alb, b.site.emis, b.site.class_idx, b.site.windcoeff};
    for (int k = 0; k < 9; ++k)
      if (!loop[k]) return fail(SW100_E_ARG, "site %d: a time-loop plane is NULL", i);
  }
  return 0;
}

}  // extern "C"

namespace {

template <class Kernel>
int launch_batch(Kernel kernel, const char* name, const sw100_batch_site* sites, const sw100_tile* tiles,
                 int n_tiles, int block_x, int block_y, int grid, void* stream) {
  int rc;
  if (n_tiles < 0) return fail(SW100_E_ARG, "n_tiles must be >= 0");
  if (n_tiles == 0) return 0;
  if ((rc = check_ptr(sites, "sites")) || (rc = check_ptr(tiles, "tiles"))) return rc;
  if (block_x <= 0 || block_y <= 0 || block_x * block_y != 128)
    return fail(SW100_E_ARG, "block %d x %d: batch kernels run 128 threads per block", block_x, block_y);
  if (grid <= 0) return fail(SW100_E_ARG, "grid must be positive");
  grid = std::min(grid, n_tiles);
  kernel<<<grid, dim3(block_x, block_y), 0, static_cast<cudaStream_t>(stream)>>>(sites, tiles, n_tiles);
  return check_launch(name);
}

}  // namespace

extern "C" {

int sw100_batch_pack(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x,
                     int block_y, int grid, void* stream) {
  return launch_batch(pack_batch_kernel, "pack_batch_kernel", sites, tiles, n_tiles, block_x, block_y, grid, stream);
}

int sw100_batch_bush_flags(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x,
                           int block_y, int grid, void* stream) {
  return launch_batch(svf_bush_flags_batch_kernel, "svf_bush_flags_batch_kernel", sites, tiles, n_tiles, block_x,
                      block_y, grid, stream);
}

int sw100_batch_skipmap(const sw100_batch_site* sites, int n_sites, void* stream) {
  int rc;
  if (n_sites < 0 || n_sites > 65535) return fail(SW100_E_ARG, "n_sites must be in [0, 65535]");
  if (n_sites == 0) return 0;
  if ((rc = check_ptr(sites, "sites"))) return rc;
  skipmap_batch_kernel<<<dim3(256, n_sites), 128, 0, static_cast<cudaStream_t>(stream)>>>(sites);
  return check_launch("skipmap_batch_kernel");
}

int sw100_batch_svf(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x, int block_y,
                    int grid, void* stream) {
  return launch_batch(svf_sweep_batch_kernel, "svf_sweep_batch_kernel", sites, tiles, n_tiles, block_x, block_y,
                      grid, stream);
}

int sw100_batch_sun_march(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x,
                          int block_y, int grid, void* stream) {
  return launch_batch(sun_march_batch_kernel, "sun_march_batch_kernel", sites, tiles, n_tiles, block_x, block_y,
                      grid, stream);
}

int sw100_batch_flux_loop(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x,
                          int block_y, int grid, void* stream) {
  return launch_batch(time_loop_batch_kernel, "time_loop_batch_kernel", sites, tiles, n_tiles, block_x, block_y,
                      grid, stream);
}

int sw100_batch_flux_loop_sums(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x,
                               int block_y, int grid, void* stream) {
  return launch_batch(time_loop_batch_sums_kernel, "time_loop_batch_sums_kernel", sites, tiles, n_tiles, block_x,
                      block_y, grid, stream);
}

int sw100_prepare_site(const float* dsm, const float* trees, const float* dem, const float* aspect_deg,
                       const float* landcover, const sw100_class_table* classes, int rows, int cols,
                       float* vegdsm, float* vegdsm2, float* bush, float* buildings, float* aspect_rad, float* tgk,
                       float* tstart, float* alb, float* emis, uint8_t* class_idx, sw100_site_stats* stats,
                       void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  const void* in[] = {dsm, trees, dem, aspect_deg, vegdsm, vegdsm2, bush, buildings, aspect_rad, tgk, tstart, alb,
                      emis, class_idx, stats};
  const char* names[] = {"dsm", "trees", "dem", "aspect_deg", "vegdsm", "vegdsm2", "bush", "buildings",
                         "aspect_rad", "tgk", "tstart", "alb", "emis", "class_idx", "stats"};
  for (int k = 0; k < 15; ++k)
    if ((rc = check_ptr(in[k], names[k]))) return rc;
  sw100_class_table table = {};
  if (landcover) {
    if ((rc = check_ptr(classes, "classes"))) return rc;
    table = *classes;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(stats, 0, sizeof(sw100_site_stats), st);
  if (e != cudaSuccess) return fail((int)e, "cudaMemsetAsync: %s", cudaGetErrorString(e));
  const size_t npix = (size_t)rows * cols;
  const int grid = (int)std::min<size_t>((npix + 255) / 256, 148 * 8);
  prepare_site_kernel<<<grid, 256, 0, st>>>(dsm, trees, dem, aspect_deg, landcover, table, npix, vegdsm, vegdsm2,
                                            bush, buildings, aspect_rad, tgk, tstart, alb, emis, class_idx, stats);
  return check_launch("prepare_site_kernel");
}

int sw100_pack_cubes(const float* shmat, const float* vegshmat, const float* vbshvegshmat, int rows, int cols,
                     int n_patches, const uint32_t* single_step, uint32_t* out_bits, void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = check_ptr(shmat, "shmat")) || (rc = check_ptr(vegshmat, "vegshmat")) ||
      (rc = check_ptr(vbshvegshmat, "vbshvegshmat")) || (rc = check_ptr(out_bits, "out_bits")))
    return rc;
  if (n_patches <= 0 || n_patches > 32 * SW100_CUBE_WORDS) return fail(SW100_E_SIZE, "n_patches out of range");
  Single5 single = {};
  if (single_step)
    for (int w = 0; w < SW100_CUBE_WORDS; ++w) single.w[w] = single_step[w];
  const size_t n = (size_t)rows * cols;
  const int threads = 256;
  const int blocks = (int)std::min<size_t>((n + threads - 1) / threads, 148 * 16);
  pack_cubes_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(shmat, vegshmat, vbshvegshmat, n,
                                                                                n_patches, single, out_bits);
  return check_launch("pack_cubes_kernel");
}

int sw100_sun_march_workspace_bytes(int rows, int cols, int64_t* bytes) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = check_ptr(bytes, "bytes"))) return rc;
  *bytes = align_up((int64_t)rows * cols * 16);
  return 0;
}

int sw100_sun_march(const sw100_site_planes* site, int rows, int cols, const sw100_series* series, float* gsrc,
                    float* debug8, void* workspace, int64_t workspace_bytes, void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = validate_site_loop(site))) return rc;
  if ((rc = validate_series(series))) return rc;
  if ((rc = check_ptr(gsrc, "gsrc"))) return rc;
  int64_t need = 0;
  if ((rc = sw100_sun_march_workspace_bytes(rows, cols, &need))) return rc;
  if ((rc = check_workspace(workspace, workspace_bytes, need))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float4* src4 = static_cast<float4*>(workspace);
  if ((rc = launch_pack(*site, rows, cols, src4, st))) return rc;
  return launch_sun_march(*site, rows, cols, *series, src4, reinterpret_cast<float4*>(gsrc), debug8, st);
}

int sw100_time_loop_workspace_bytes(int rows, int cols, int n_day, int64_t* bytes) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = check_ptr(bytes, "bytes"))) return rc;
  if (n_day < 0) return fail(SW100_E_ARG, "n_day must be >= 0");
  const int64_t plane4 = align_up((int64_t)rows * cols * 16);
  *bytes = plane4 * (1 + (int64_t)n_day);
  return 0;
}

int sw100_time_loop(const sw100_site_planes* site, int rows, int cols, const sw100_series* series, float* state,
                    uint32_t out_mask, float* outputs, void* workspace, int64_t workspace_bytes, void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = validate_site_loop(site))) return rc;
  if ((rc = validate_series(series))) return rc;
  if ((rc = check_ptr(state, "state"))) return rc;
  if (out_mask & ~0x7Fu) return fail(SW100_E_ARG, "unknown output bits 0x%x", out_mask);
  if (out_mask && !outputs) return fail(SW100_E_ARG, "outputs must not be NULL");
  int64_t need = 0;
  if ((rc = sw100_time_loop_workspace_bytes(rows, cols, series->n_day, &need))) return rc;
  if ((rc = check_workspace(workspace, workspace_bytes, need))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t plane4 = align_up((int64_t)rows * cols * 16);
  float4* src4 = static_cast<float4*>(workspace);
  float4* gsrc = reinterpret_cast<float4*>(static_cast<char*>(workspace) + plane4);
  if ((rc = launch_pack(*site, rows, cols, src4, st))) return rc;
  if ((rc = launch_sun_march(*site, rows, cols, *series, src4, gsrc, nullptr, st))) return rc;
  dim3 block, grid;
  if ((rc = loop_shape(*site, rows, cols, grid, block))) return rc;
  time_loop_kernel<<<grid, block, 0, st>>>(make_site(*site), rows, cols, series->steps, series->n_t, series->patch,
                                           series->n_patches, series->gvf, gsrc, series->n_day, state, out_mask,
                                           outputs);
  return check_launch("time_loop_kernel");
}

int sw100_flux_loop(const sw100_site_planes* site, int rows, int cols, const sw100_series* series, const float* gsrc,
                    float* state, uint32_t out_mask, float* outputs, void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = validate_site_loop(site))) return rc;
  if ((rc = validate_series(series))) return rc;
  if ((rc = check_ptr(state, "state"))) return rc;
  if (series->n_day > 0 && (rc = check_ptr(gsrc, "gsrc"))) return rc;
  if (out_mask & ~0x7Fu) return fail(SW100_E_ARG, "unknown output bits 0x%x", out_mask);
  if (out_mask && !outputs) return fail(SW100_E_ARG, "outputs must not be NULL");
  dim3 block, grid;
  if ((rc = loop_shape(*site, rows, cols, grid, block))) return rc;
  time_loop_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      make_site(*site), rows, cols, series->steps, series->n_t, series->patch, series->n_patches, series->gvf,
      reinterpret_cast<const float4*>(gsrc), series->n_day, state, out_mask, outputs);
  return check_launch("time_loop_kernel");
}

int sw100_patch_sums_workspace_bytes(int n_t, int64_t* bytes) {
  int rc;
  if ((rc = check_ptr(bytes, "bytes"))) return rc;
  if (n_t < 0) return fail(SW100_E_ARG, "n_t must be >= 0");
  *bytes = align_up((int64_t)((n_t + 7) / 8) * 96 * 624 * 2);
  return 0;
}

int sw100_patch_sums(const sw100_site_planes* site, int rows, int cols, const sw100_series* series, float* sums,
                     int32_t* err, void* workspace, int64_t workspace_bytes, void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = validate_site_loop(site))) return rc;
  if ((rc = validate_series(series))) return rc;
  if ((rc = check_ptr(sums, "sums"))) return rc;
  if (series->n_patches > 156) return fail(SW100_E_ARG, "at most 156 patches (n_patches %d)", series->n_patches);
  int64_t need = 0;
  if ((rc = sw100_patch_sums_workspace_bytes(series->n_t, &need))) return rc;
  if ((rc = check_workspace(workspace, workspace_bytes, need))) return rc;
  if (series->n_t == 0) return 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int n_groups = (series->n_t + 7) / 8;
  __nv_bfloat16* W = static_cast<__nv_bfloat16*>(workspace);
  const int64_t nw = (int64_t)n_groups * 96 * 624;
  patch_weights_kernel<<<(unsigned)std::min<int64_t>((nw + 255) / 256, 148 * 8), 256, 0, st>>>(
      series->steps, series->n_t, series->patch, series->n_patches, W, n_groups);
  if ((rc = check_launch("patch_weights_kernel"))) return rc;
  // three stages of A (12 KB) and B (9 KB) chunks: 63 KB, at most 3 CTAs
  // (3 x 128 TMEM columns) per SM
  const int smem = 3 * (12288 + 9216);
  // the attributes are per function and process: set them once (the largest
  // shared-memory carveout, so that several 56 KB CTAs share an SM)
  static std::once_flag attr_once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(attr_once, [&] {
    attr_err = cudaFuncSetAttribute(patch_sums_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (attr_err == cudaSuccess)
      attr_err = cudaFuncSetAttribute(patch_sums_tc_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      (int)cudaSharedmemCarveoutMaxShared);
  });
  if (attr_err != cudaSuccess) return fail((int)attr_err, "cudaFuncSetAttribute: %s", cudaGetErrorString(attr_err));
  const int64_t npix = (int64_t)rows * cols;
  patch_sums_tc_kernel<<<(unsigned)((npix + 127) / 128), 128, smem, st>>>(
      site->bits, npix, series->n_patches, W, n_groups, series->n_t, sums, err, g_tc_wait_limit.load());
  return check_launch("patch_sums_tc_kernel");
}

int sw100_walk_work(const sw100_site_planes* site, int rows, int cols, const sw100_gvf_azimuth* gvf, int second,
                    int32_t* work, void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = check_ptr(site, "site")) || (rc = check_ptr(site->buildings, "buildings")) ||
      (rc = check_ptr(gvf, "gvf")) || (rc = check_ptr(work, "work")))
    return rc;
  if (second < 0 || second > SW100_MAX_GVF_STEPS)
    return fail(SW100_E_ARG, "second %d outside 0 .. %d", second, SW100_MAX_GVF_STEPS);
  const int64_t n = (int64_t)((rows + 3) / 4) * ((cols + 7) / 8);
  const int64_t threads = n * 32;
  walk_work_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
      site->buildings, rows, cols, gvf, second, work, (int)n);
  return check_launch("walk_work_kernel");
}

int sw100_flux_loop_sums(const sw100_site_planes* site, int rows, int cols, const sw100_series* series,
                         const float* gsrc, const float* sums, float* state, uint32_t out_mask, float* outputs,
                         void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = validate_site_loop(site))) return rc;
  if ((rc = validate_series(series))) return rc;
  if ((rc = check_ptr(state, "state")) || (rc = check_ptr(sums, "sums"))) return rc;
  if (series->n_day > 0 && (rc = check_ptr(gsrc, "gsrc"))) return rc;
  if (out_mask & ~0x7Fu) return fail(SW100_E_ARG, "unknown output bits 0x%x", out_mask);
  if (out_mask && !outputs) return fail(SW100_E_ARG, "outputs must not be NULL");
  // six 33 KB blocks per SM (the register bound) need the largest
  // shared-memory carveout; set once per process
  static std::once_flag attr_once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(attr_once, [&] {
    attr_err = cudaFuncSetAttribute(time_loop_sums_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared);
  });
  if (attr_err != cudaSuccess) return fail((int)attr_err, "cudaFuncSetAttribute: %s", cudaGetErrorString(attr_err));
  dim3 block, grid;
  if ((rc = loop_shape(*site, rows, cols, grid, block))) return rc;
  time_loop_sums_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      make_site(*site), rows, cols, series->steps, series->n_t, series->patch, series->n_patches, series->gvf,
      reinterpret_cast<const float4*>(gsrc), series->n_day, state, out_mask, outputs, sums);
  return check_launch("time_loop_sums_kernel");
}

int sw100_utci(const float* ta, const float* rh, const float* tmrt, const float* va, int64_t n, float* out,
               void* stream) {
  int rc;
  if (n < 0) return fail(SW100_E_ARG, "n must be >= 0");
  if (n == 0) return 0;
  if ((rc = check_ptr(ta, "ta")) || (rc = check_ptr(rh, "rh")) || (rc = check_ptr(tmrt, "tmrt")) ||
      (rc = check_ptr(va, "va")) || (rc = check_ptr(out, "out")))
    return rc;
  const int threads = 256;
  const int blocks = (int)std::min<int64_t>((n + threads - 1) / threads, 148 * 32);
  utci_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(ta, rh, tmrt, va, n, out);
  return check_launch("utci_kernel");
}

}  // extern "C"

// ------------------------------------------------- allocation-free variant
// Scratch of sw100_svf_sweep_noalloc: a file-scope device array, one per
// device that loads the library.  Host code must not use its name as a
// device address; the address is looked up per device below.
namespace {
__device__ __align__(256) unsigned char g_svf_noalloc_scratch[SW100_SVF_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 128;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up with
// that device current on the first call for it and cached (the cache is not
// refreshed after cudaDeviceReset; see the header).
int noalloc_scratch(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail((int)e, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(SW100_E_ARG, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_svf_noalloc_scratch);
    if (e != cudaSuccess) return fail((int)e, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return 0;
}
}  // namespace

extern "C" int sw100_svf_sweep_noalloc(const sw100_site_planes* site, int rows, int cols, const sw100_svf_plan* plan,
                                       const sw100_step* steps, int n_steps, float* out_planes, uint32_t* out_bits,
                                       void* stream) {
  int rc;
  int64_t need = 0;
  if ((rc = sw100_svf_workspace_bytes(rows, cols, n_steps, &need))) return rc;
  if (need > (int64_t)SW100_SVF_NOALLOC_SCRATCH_BYTES)
    return fail(SW100_E_SIZE,
                "grid %d x %d with %d steps needs %lld scratch bytes; the allocation-free sweep has %lld "
                "(at most 1024 x 1024 pixels)",
                rows, cols, n_steps, (long long)need, (long long)SW100_SVF_NOALLOC_SCRATCH_BYTES);
  if ((rc = validate_site_march(site))) return rc;
  if ((rc = check_ptr(plan, "plan")) || (rc = check_ptr(steps, "steps")) || (rc = check_ptr(out_planes, "out_planes")) ||
      (rc = check_ptr(out_bits, "out_bits")))
    return rc;
  void* scratch = nullptr;
  if ((rc = noalloc_scratch(&scratch))) return rc;
  // the workspace sweep's own launches (packing, bush flags, skip map,
  // sweep), with the static array as its workspace
  return run_svf_sweep(site, rows, cols, plan, steps, n_steps, out_planes, out_bits, scratch,
                       (int64_t)SW100_SVF_NOALLOC_SCRATCH_BYTES, nullptr, stream);
}

extern "C" int sw100_utci_steps(const sw100_time_step* steps, int n_steps, const float* tmrt,
                                const float* buildings, const float* windcoeff, int64_t npix, float* out,
                                void* stream) {
  int rc;
  if (n_steps < 0 || npix < 0) return fail(SW100_E_ARG, "n_steps and npix must be >= 0");
  if (n_steps == 0 || npix == 0) return 0;
  if ((rc = check_ptr(steps, "steps")) || (rc = check_ptr(tmrt, "tmrt")) || (rc = check_ptr(buildings, "buildings")) ||
      (rc = check_ptr(out, "out")))
    return rc;
  const int threads = 256;
  const int bx = (int)std::min<int64_t>((npix + threads - 1) / threads, 148 * 4);
  const dim3 grid(bx, std::min(n_steps, 65535));
  utci_steps_kernel<<<grid, threads, 0, static_cast<cudaStream_t>(stream)>>>(steps, n_steps, tmrt, buildings,
                                                                             windcoeff, npix, out);
  return check_launch("utci_steps_kernel");
}

// ------------------------------------------------------------ learned preview
namespace {

int check_act(int N, int H, int W, int C, int stride, int coff, const char* what) {
  if (N <= 0 || H <= 0 || W <= 0 || C <= 0) return fail(SW100_E_SIZE, "%s: empty tensor", what);
  if (C % 16 || stride % 16 || coff % 16 || coff + C > stride)
    return fail(SW100_E_ARG, "%s: channels %d at offset %d of %d must be multiples of 16 inside the stride", what, C,
                coff, stride);
  if ((int64_t)N * H * W * stride >= (int64_t)1 << 31) return fail(SW100_E_SIZE, "%s: tensor too large", what);
  return 0;
}

int grid1(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }

}  // namespace

extern "C" {

int sw100_nn_conv3x3_tc(const void* x, int n, int h, int w, int cin, int xstride, int xcoff, const void* wt,
                        const float* bias, int cout, void* y, int ystride, int ycoff, int relu, int out_f32,
                        int32_t* err, void* stream) {
  int rc;
  if ((rc = check_ptr(x, "x")) || (rc = check_ptr(wt, "wt")) || (rc = check_ptr(y, "y"))) return rc;
  if ((rc = check_act(n, h, w, cin, xstride, xcoff, "x")) || (rc = check_act(n, h, w, cout, ystride, ycoff, "y")))
    return rc;
  if (cout > 128) return fail(SW100_E_ARG, "the tensor-core convolution takes at most 128 output channels");
  const int64_t total = (int64_t)n * h * w;
  const int64_t blocks = (total + 127) / 128;
  // three stages of A tiles (4 K steps x 128 pixels x 32 B) and of B tiles
  // (4 K steps x cout x 32 B): the fewer the output channels, the more CTAs
  // share an SM
  const int smem = 3 * 4 * 4096 + 3 * 4 * 32 * cout;
  static bool attr_set = false;    // the attribute is per function and process: set it once, to the largest size
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(nn_conv3x3_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         3 * 4 * 4096 + 3 * 4 * 32 * 128);
    if (e != cudaSuccess) return fail((int)e, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    attr_set = true;
  }
  nn_conv3x3_tc_kernel<<<(unsigned)blocks, 128, smem, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(x), n, h, w, cin, xstride, xcoff, static_cast<const __nv_bfloat16*>(wt), bias,
      cout, y, ystride, ycoff, relu, out_f32, err, g_tc_wait_limit.load());
  return check_launch("nn_conv3x3_tc_kernel");
}

int sw100_set_wait_limit(int polls) {
  const int prev = g_tc_wait_limit.load();
  g_tc_wait_limit.store(polls < 0 ? kDefaultTcWaitLimit : polls);
  return prev;
}

int sw100_nn_conv3x3_wgrad(const void* x, int n, int h, int w, int cin, int xstride, int xcoff, const void* dy,
                           int cout, int dstride, int dcoff, float* dw, float* dbias, void* stream) {
  int rc;
  if ((rc = check_ptr(x, "x")) || (rc = check_ptr(dy, "dy")) || (rc = check_ptr(dw, "dw"))) return rc;
  if ((rc = check_act(n, h, w, cin, xstride, xcoff, "x")) || (rc = check_act(n, h, w, cout, dstride, dcoff, "dy")))
    return rc;
  const int rows = n * h;
  const int rows_per_block = std::max(1, rows / 148);
  dim3 grid((rows + rows_per_block - 1) / rows_per_block, 9, ((cout + 63) / 64) * ((cin + 63) / 64));
  nn_wgrad_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(x), n, h, w, cin, xstride, xcoff, static_cast<const __nv_bfloat16*>(dy), cout,
      dstride, dcoff, dw, dbias, rows_per_block);
  return check_launch("nn_wgrad_kernel");
}

int sw100_nn_weights(const float* master, int cin, int cout, void* wf, void* wd, void* stream) {
  int rc;
  if ((rc = check_ptr(master, "master")) || (rc = check_ptr(wf, "wf"))) return rc;
  if (cin <= 0 || cout <= 0 || cin % 16 || cout % 16) return fail(SW100_E_ARG, "channels must be multiples of 16");
  nn_weights_kernel<<<grid1(9 * cin * cout), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      master, cin, cout, static_cast<__nv_bfloat16*>(wf), static_cast<__nv_bfloat16*>(wd));
  return check_launch("nn_weights_kernel");
}

int sw100_nn_relu_bwd(void* dy, const void* y, int64_t npix, int c, int dstride, int dcoff, int ystride, int ycoff,
                      void* stream) {
  int rc;
  if ((rc = check_ptr(dy, "dy")) || (rc = check_ptr(y, "y"))) return rc;
  if (npix <= 0 || c <= 0 || dcoff + c > dstride || ycoff + c > ystride) return fail(SW100_E_ARG, "bad relu extents");
  nn_relu_bwd_kernel<<<grid1(npix * c), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<__nv_bfloat16*>(dy), static_cast<const __nv_bfloat16*>(y), npix, c, dstride, dcoff, ystride, ycoff);
  return check_launch("nn_relu_bwd_kernel");
}

int sw100_nn_pool2(const void* x, int n, int h, int w, int c, int xstride, int xcoff, void* y, int ystride, int ycoff,
                   int backward, int accumulate, void* stream) {
  int rc;
  if ((rc = check_ptr(x, "x")) || (rc = check_ptr(y, "y"))) return rc;
  if (h % 2 || w % 2) return fail(SW100_E_ARG, "pooling needs even sizes");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!backward) {
    if ((rc = check_act(n, h, w, c, xstride, xcoff, "x")) || (rc = check_act(n, h / 2, w / 2, c, ystride, ycoff, "y")))
      return rc;
    nn_pool2_kernel<<<grid1((int64_t)n * h * w * c / 4), 256, 0, st>>>(static_cast<const __nv_bfloat16*>(x), n, h, w, c,
                                                                        xstride, xcoff, static_cast<__nv_bfloat16*>(y),
                                                                        ystride, ycoff);
    return check_launch("nn_pool2_kernel");
  }
  // backward: x = dY (h/2 x w/2), y = dX (h x w)
  if ((rc = check_act(n, h / 2, w / 2, c, xstride, xcoff, "dy")) || (rc = check_act(n, h, w, c, ystride, ycoff, "dx")))
    return rc;
  nn_pool2_bwd_kernel<<<grid1((int64_t)n * h * w * c), 256, 0, st>>>(static_cast<const __nv_bfloat16*>(x), n, h, w, c,
                                                                      xstride, xcoff, static_cast<__nv_bfloat16*>(y),
                                                                      ystride, ycoff, accumulate);
  return check_launch("nn_pool2_bwd_kernel");
}

int sw100_nn_up2(const void* x, int n, int h, int w, int c, int xstride, int xcoff, void* y, int ystride, int ycoff,
                 int backward, void* stream) {
  int rc;
  if ((rc = check_ptr(x, "x")) || (rc = check_ptr(y, "y"))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!backward) {
    if ((rc = check_act(n, h, w, c, xstride, xcoff, "x")) || (rc = check_act(n, 2 * h, 2 * w, c, ystride, ycoff, "y")))
      return rc;
    nn_up2_kernel<<<grid1((int64_t)n * 4 * h * w * c), 256, 0, st>>>(static_cast<const __nv_bfloat16*>(x), n, h, w, c,
                                                                      xstride, xcoff, static_cast<__nv_bfloat16*>(y),
                                                                      ystride, ycoff);
    return check_launch("nn_up2_kernel");
  }
  // backward: x = dY (2h x 2w), y = dX (h x w)
  if ((rc = check_act(n, 2 * h, 2 * w, c, xstride, xcoff, "dy")) || (rc = check_act(n, h, w, c, ystride, ycoff, "dx")))
    return rc;
  nn_up2_bwd_kernel<<<grid1((int64_t)n * h * w * c), 256, 0, st>>>(static_cast<const __nv_bfloat16*>(x), n, h, w, c,
                                                                    xstride, xcoff, static_cast<__nv_bfloat16*>(y),
                                                                    ystride, ycoff);
  return check_launch("nn_up2_bwd_kernel");
}

int sw100_nn_mse(const float* pred, const float* target, int n, int h, int w, int c, int nc, int margin, void* dpred,
                 float* loss, void* stream) {
  int rc;
  if ((rc = check_ptr(pred, "pred")) || (rc = check_ptr(target, "target"))) return rc;
  if (n <= 0 || h <= 2 * margin || w <= 2 * margin || nc <= 0 || nc > c || margin < 0)
    return fail(SW100_E_ARG, "bad loss extents");
  const float inv = 1.f / ((float)n * (h - 2 * margin) * (w - 2 * margin) * nc);
  nn_mse_kernel<<<grid1((int64_t)n * h * w * c), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      pred, target, n, h, w, c, nc, margin, inv, static_cast<__nv_bfloat16*>(dpred), loss);
  return check_launch("nn_mse_kernel");
}

int sw100_nn_adam(float* param, const float* grad, float* m, float* v, int64_t n, float lr, float b1, float b2,
                  float eps, int step, void* stream) {
  int rc;
  if ((rc = check_ptr(param, "param")) || (rc = check_ptr(grad, "grad")) || (rc = check_ptr(m, "m")) ||
      (rc = check_ptr(v, "v")))
    return rc;
  if (n <= 0 || step <= 0) return fail(SW100_E_ARG, "n and step must be positive");
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  nn_adam_kernel<<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(param, grad, m, v, n, lr, b1, b2, eps, c1, c2);
  return check_launch("nn_adam_kernel");
}

int sw100_nn_input(const float* dsm, const float* vegdsm, const float* vegdsm2, const float* dem, int rows, int cols,
                   const int32_t* origins, int n, int size, void* x, void* stream) {
  int rc;
  if ((rc = check_grid(rows, cols))) return rc;
  if ((rc = check_ptr(dsm, "dsm")) || (rc = check_ptr(vegdsm, "vegdsm")) || (rc = check_ptr(vegdsm2, "vegdsm2")) ||
      (rc = check_ptr(origins, "origins")) || (rc = check_ptr(x, "x")))
    return rc;
  if (n <= 0 || size <= 0) return fail(SW100_E_ARG, "n and size must be positive");
  nn_input_kernel<<<grid1((int64_t)n * size * size), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dsm, vegdsm, vegdsm2, dem, rows, cols, reinterpret_cast<const int2*>(origins), n, size,
      static_cast<__nv_bfloat16*>(x));
  return check_launch("nn_input_kernel");
}

}  // extern "C"


// ------------------------------------------------------------ march tables
// Host-side step tables of the SVF patch marches (shadow.py:196-247) and the
// sun march (solweig.py:1092-1149).  Every float32 operation is rounded on
// its own: this file is compiled without floating-point contraction.
namespace {

struct MarchStep {
  float dx, dy, dz;
};

inline MarchStep march_step(const sw100_march_const& m, float fi) {
  MarchStep s;
  const float m_scos = -1.f * m.scos;
  if (m.branch_y) {
    s.dy = m.ssin * fi;
    s.dx = m_scos * std::fabs(std::nearbyint(fi / m.tan_a));
  } else {
    s.dy = m.ssin * std::fabs(std::nearbyint(fi * m.tan_a));
    s.dx = m_scos * fi;
  }
  s.dz = (m.ds * fi) * m.tanalt;
  return s;
}

// float32 -> int32 as x86-64's truncating conversion: INT32_MIN for NaN,
// infinities and values outside the int32 range
inline int32_t to_i32(float v) {
  if (!(v > -2147483904.f && v < 2147483648.f)) return INT32_MIN;
  return (int32_t)v;
}

inline bool step_ok(const MarchStep& s, float amax, int rows, int cols) {
  return amax >= s.dz && std::fabs(s.dx) < (float)rows && std::fabs(s.dy) < (float)cols;
}

// SW100_STEP_SKIP8 of one march's n executed steps: step k >= 1 when no step
// k+1 .. k+7 moves more than one cell per axis from the step before it and
// dz does not decrease (NaN counts as a decrease) over the steps k .. k+7
// compared with their predecessors.
void skip_flags(sw100_step* t, int64_t n) {
  if (n <= 0) return;
  t[0].flags = 0;
  int64_t next_mv = INT64_MAX, next_dz = INT64_MAX;  // nearest faulty step >= k + 1 / >= k
  for (int64_t k = n - 1; k >= 1; --k) {
    if (k + 1 < n) {
      const int64_t ddx = (int64_t)t[k + 1].dx - t[k].dx, ddy = (int64_t)t[k + 1].dy - t[k].dy;
      if (ddx > 1 || ddx < -1 || ddy > 1 || ddy < -1) next_mv = k + 1;
    }
    if (!(t[k].dz >= t[k - 1].dz)) next_dz = k;
    t[k].flags = (next_mv > k + 7 && next_dz > k + 7) ? SW100_STEP_SKIP8 : 0;
  }
}

}  // namespace

extern "C" int sw100_march_tables(const sw100_march_const* marches, int n_marches, int first_index, float amax,
                                  int rows, int cols, sw100_step* steps, int64_t capacity, int32_t* counts,
                                  int64_t* total) {
  int rc;
  if ((rc = check_grid(rows, cols)) || (rc = check_ptr(counts, "counts")) || (rc = check_ptr(total, "total")))
    return rc;
  if (n_marches < 0 || (n_marches > 0 && !marches)) return fail(SW100_E_ARG, "marches must hold n_marches >= 0 entries");
  if (first_index < 0) return fail(SW100_E_ARG, "first_index must be >= 0");
  const int last = std::max(rows, cols) + 2;
  const int64_t len = last >= first_index ? (int64_t)last - first_index + 1 : 0;
  int64_t sum = 0;
  if (steps && capacity >= (int64_t)n_marches * len) {
    // room for every march at full length: count and fill in one pass, each
    // march's steps written where the packed table puts them
    sw100_step* t = steps;
    for (int q = 0; q < n_marches; ++q) {
      int64_t n = 0;
      if (amax >= 0.f) {
        n = len;
        for (int64_t j = 0; j < len; ++j) {
          const MarchStep s = march_step(marches[q], (float)(first_index + j));
          t[j].dx = to_i32(s.dx);
          t[j].dy = to_i32(s.dy);
          t[j].dz = s.dz;
          if (!step_ok(s, amax, rows, cols)) {
            n = j + 1;
            break;
          }
        }
      }
      counts[q] = (int32_t)n;
      skip_flags(t, n);
      t += n;
      sum += n;
    }
    *total = sum;
    return 0;
  }
  for (int q = 0; q < n_marches; ++q) {
    int64_t n = 0;
    if (amax >= 0.f) {
      n = len;
      for (int64_t j = 0; j < len; ++j) {
        if (!step_ok(march_step(marches[q], (float)(first_index + j)), amax, rows, cols)) {
          n = j + 1;
          break;
        }
      }
    }
    counts[q] = (int32_t)n;
    sum += n;
  }
  *total = sum;
  if (!steps) return 0;
  if (sum > capacity)
    return fail(SW100_E_WORKSPACE, "%lld steps do not fit a table of %lld", (long long)sum, (long long)capacity);
  sw100_step* t = steps;
  for (int q = 0; q < n_marches; ++q) {
    for (int64_t j = 0; j < counts[q]; ++j) {
      const MarchStep s = march_step(marches[q], (float)(first_index + j));
      t[j].dx = to_i32(s.dx);
      t[j].dy = to_i32(s.dy);
      t[j].dz = s.dz;
    }
    skip_flags(t, counts[q]);
    t += counts[q];
  }
  return 0;
}
