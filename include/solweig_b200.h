/*
 * solweig_b200.h -- C ABI of the B200 (sm_100a) SOLWEIG radiation chain.
 *
 * Plain C: pointers, sizes and POD tables.  Every entry point returns 0 on
 * success or a non-zero status (a CUDA error code, or SW100_E_* below); the
 * message of the last failure on the calling thread is available from
 * sw100_last_error().  No entry point aborts the process, and none allocates
 * device memory: scratch space is a caller-provided `workspace` whose size
 * the matching *_workspace_bytes() query returns.
 *
 * Memory: unless a parameter is documented as a host pointer, array
 * arguments are DEVICE pointers on the current device.  Rasters are
 * row-major float32 (rows, cols), npix = rows * cols.  Patch bit cubes are
 * word-planar: word w of pixel i of cube k lives at
 * bits[(k * SW100_CUBE_WORDS + w) * npix + i]; bit (p & 31) of word (p >> 5)
 * is patch p.  `stream` is a cudaStream_t (NULL = legacy default stream).
 *
 * Reference interfaces replaced (paths inside Synn-Arch/Solweig_Project):
 *   sw100_svf_sweep   <- solweig_gpu/shadow.py:409-625 svf_calculator, with
 *                        shadow.py:166-322 shadow() for each patch; native
 *                        counterpart native/cuda/src/sw_api.cu:209-250
 *                        (sw_run_march_svf_shadow per patch + sw_run_fold)
 *   sw100_sun_march   <- solweig_gpu/solweig.py:1079-1224
 *                        shadowingfunction_wallheight_23 (one call per
 *                        daytime step); native counterpart
 *                        native/cuda/src/sw_api.cu:218-228
 *                        (sw_run_march_wallheight23)
 *   sw100_time_loop   <- solweig_gpu/utci_process.py:917-1067, the time loop
 *                        of run_utci_window around Solweig_2022a_calc
 *                        (solweig_gpu/solweig.py:1950-2311) and
 *                        utci_calculator; native counterpart
 *                        native/cuda/src/sw_api.cu:253-344 (sw_run_rad_day,
 *                        sw_run_rad_night, sw_utci_*)
 *   sw100_utci        <- solweig_gpu/calculate_utci.py:259-330 utci_calculator;
 *                        native counterpart native/cuda/src/sw_api.cu:327-344
 *   sw100_abi_version, sw100_last_error
 *                     <- native/cuda/src/sw_api.cu:29-37 (sw_last_error,
 *                        sw_abi_version)
 */
#ifndef SOLWEIG_B200_H
#define SOLWEIG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SW100_ABI_VERSION 3

#define SW100_MAX_PATCHES 160   /* patch option 2 uses 153 */
#define SW100_MAX_RINGS 16
#define SW100_MAX_ANNULI 16     /* annuli per altitude band (12 in option 2) */
#define SW100_CUBE_WORDS 5      /* ceil(153 / 32) */
#define SW100_MAX_CLASSES 8     /* land-cover property classes */
#define SW100_N_GVF_AZ 18       /* ground view factor search azimuths */
#define SW100_UTCI_TERMS 210   /* terms of the UTCI regression */
#define SW100_MAX_GVF_STEPS 64  /* bound on the `second` walk length */
#define SW100_SVF_PLANES 19     /* 15 SVF planes, SVFtotal, 3 time-loop statics */

/* status codes beyond CUDA's */
#define SW100_E_ARG 1001         /* invalid argument */
#define SW100_E_SIZE 1002        /* size outside the supported range */
#define SW100_E_WORKSPACE 1003   /* workspace missing or too small */

/* One executed step of a march: source offset (dx rows, dy cols) and the
 * float32 height drop dz, built on the host with the reference's float32
 * trigonometry so that the executed sequence is bit-identical.  flags bit 0
 * (SW100_STEP_SKIP8) is the host's proof that steps k .. k+7 of the same march
 * (those that exist) each move at most one cell per axis from the step
 * before and that dz does not decrease from step k-1 through k+7: the
 * kernels then may test those 8 steps at once against a coarse height bound
 * (an exact shortcut).  0 is always valid. */
#define SW100_STEP_SKIP8 1
typedef struct {
  int32_t dx;
  int32_t dy;
  float dz;
  int32_t flags;
} sw100_step;

/* ------------------------------------------------------ march tables -- */
/* Float32 constants of one march direction: the SVF patch marches of
 * svf_calculator (shadow.py:196-226) and the sun march of
 * shadowingfunction_wallheight_23 (solweig.py:1092-1120).  branch_y: the
 * step walks the y axis by one cell (azimuth in [pi/4, 3pi/4) or
 * [5pi/4, 7pi/4)); ssin / scos: sign(sin az), sign(cos az); tan_a: tan az;
 * ds: |1 / sin az| when branch_y, else |1 / cos az|; tanalt: tan(alt) / scale. */
typedef struct {
  int32_t branch_y;
  float ssin;
  float scos;
  float tan_a;
  float ds;
  float tanalt;
} sw100_march_const;

/* Executed steps of n_marches marches (host only, no device work).  Step
 * index i runs over first_index .. max(rows, cols) + 2 (1 for the SVF
 * patches, 0 for the sun march) with, in float32, one rounding per
 * operation:
 *   branch_y: dy = ssin * i, dx = (-1 * scos) * |rint(i / tan_a)|
 *   else:     dy = ssin * |rint(i * tan_a)|, dx = (-1 * scos) * i
 *   dz = (ds * i) * tanalt
 * A march executes its steps up to and including the first one that fails
 * amax >= dz, |dx| < rows, |dy| < cols (none when amax >= 0 fails): the
 * reference's while loop tests the previous step's values.  counts[k] (n_marches
 * entries) receives each march's step count and *total their sum; when
 * `steps` is not NULL the steps are written there concatenated in march
 * order (dx, dy converted to int32 as a C cast on x86-64 does, INT32_MIN
 * for a non-finite or out-of-range value) with their SW100_STEP_SKIP8
 * flags, refused with SW100_E_WORKSPACE when *total exceeds `capacity`.
 * Replaces the numpy loop of tables.svf_plan / tables.sun_tables. */
int sw100_march_tables(const sw100_march_const* marches, int n_marches, int first_index, float amax, int rows,
                       int cols, sw100_step* steps, int64_t capacity, int32_t* counts, int64_t* total);

/* ------------------------------------------------------- site planes -- */
/* Per-site rasters (device pointers, npix each unless noted). */
typedef struct {
  const float* dsm;          /* building DSM `a` */
  const float* vegdsm;       /* canopy top (trees + dsm, 0 where no tree) */
  const float* vegdsm2;      /* trunk zone top (0.25 trees + dsm) */
  const float* bush;         /* may be NULL when all zero */
  float vmax;                /* max over dsm, vegdsm, vegdsm2 (march early exit) */
  int32_t bush_any;          /* bush.max() > 0 */
  /* time-loop statics */
  const float* svfbuveg;     /* svf - (1 - svfveg) * (1 - transVeg) */
  const float* hsvf;         /* tan(acos(sqrt(svf))), float32 as the reference rounds it */
  const float* tan_alfa;     /* tan(svfalfa), svfalfa = asin(exp(log(1 - tmp) / 2)) */
  const float* buildings;    /* 1 ground, 0 building (dsm - dem < 2) */
  const float* walls;        /* wall height */
  const float* aspect_rad;   /* wall aspect * pi / 180 */
  const float* tgk;          /* land-cover TgK, Tstart, albedo, emissivity */
  const float* tstart;
  const float* alb;
  const float* emis;
  const uint8_t* class_idx;  /* index into sw100_time_step.tg_factor per pixel */
  const float* windcoeff;
  const uint32_t* bits;      /* 3 cubes from sw100_svf_sweep: sh, vegsh, vbshvegsh */
  /* patches whose SVF march ran at most one step: there vbshvegsh is 1 or 2
   * and its cube bit means "vbshvegsh == 1"; elsewhere it means "!= 0" */
  uint32_t single_step[SW100_CUBE_WORDS];
  /* Optional order of the time / flux loops' work (NULL: 8 x 16 blocks in
   * grid order).  The loops then run 128-thread blocks of four 8 x 4 pixel
   * patches, one per warp, taken from this list in order; patch k covers
   * rows 4 (k / pc) .. + 3 and columns 8 (k % pc) .. + 7, pc = ceil(cols / 8).
   * n_patch_order must be ceil(rows / 4) * pc and the list a permutation of
   * 0 .. n_patch_order - 1 (entries outside that range compute nothing; a
   * repeated or missing patch computes a pixel twice or not at all).  The
   * per-patch ground-view walk work of sw100_walk_work sorted descending
   * gives blocks whose warps walk alike.  Results do not depend on it. */
  const int32_t* patch_order;
  int32_t n_patch_order;
} sw100_site_planes;

/* ------------------------------------------------- site preparation -- */
/* Maxima the host needs after sw100_prepare_site, by index into
 * sw100_site_stats.max_key. */
#define SW100_STAT_DSM 0          /* dsm */
#define SW100_STAT_VEGDEM 1       /* canopy (clipped at 0) + dem: amaxvalue with the dsm maximum */
#define SW100_STAT_VEGDSM 2       /* vegdsm, vegdsm2: the march bound with the dsm maximum */
#define SW100_STAT_VEGDSM2 3
#define SW100_STAT_ABS_DSM 4      /* |dsm|, |vegdsm|, |vegdsm2| */
#define SW100_STAT_ABS_VEGDSM 5
#define SW100_STAT_ABS_VEGDSM2 6
#define SW100_STAT_BUSH 7         /* bush: the bush flag is "maximum > 0" */
#define SW100_N_SITE_STATS 8

/* Reductions of sw100_prepare_site (device memory, cleared by the call).
 * A maximum x is stored as its order-preserving key k: k = bits | 2^31
 * for x >= +0, k = ~bits for x <= -0 (so -0 < +0); NaN inputs set their
 * bit in nan_mask instead, and the maximum is then NaN, as numpy's is. */
typedef struct {
  uint32_t max_key[SW100_N_SITE_STATS];
  uint32_t nan_mask;        /* bit s: maximum s met a NaN */
  uint32_t nonfinite;       /* a NaN or infinity in dsm, vegdsm or vegdsm2 */
  uint32_t codes;           /* bit c: cleaned land-cover code c (1..7) occurs */
  uint32_t bad_codes;       /* a cleaned land-cover value has no class row */
} sw100_site_stats;

/* Land-cover classes by cleaned code 1..7 (landcoverclasses_2016a rows):
 * float32 TgK, Tstart, albedo, emissivity; bit c of `valid` set when code c
 * has exactly one class row. */
typedef struct {
  float tgk[8];
  float tstart[8];
  float alb[8];
  float emis[8];
  uint32_t valid;
} sw100_class_table;

/* The rasters the chain derives from a site's inputs, all on the device in
 * one pass (replaces the host preparation of utci_process.py:667-681,
 * :733-766, :1377-1385 and solweig.py:2083): vegdsm, vegdsm2, bush,
 * buildings, aspect in radians, the land-cover property planes and per
 * pixel the cleaned land-cover code (class_idx; 0 without land cover), plus
 * the maxima of sw100_site_stats.  Inputs and outputs are npix device
 * planes; `landcover` may be NULL (default properties), `classes` is a host
 * pointer, required with land cover. */
int sw100_prepare_site(const float* dsm, const float* trees, const float* dem, const float* aspect_deg,
                       const float* landcover, const sw100_class_table* classes, int rows, int cols,
                       float* vegdsm, float* vegdsm2, float* bush, float* buildings, float* aspect_rad, float* tgk,
                       float* tstart, float* alb, float* emis, uint8_t* class_idx, sw100_site_stats* stats,
                       void* stream);

/* ---------------------------------------------------------------- SVF -- */
typedef struct {
  int32_t n_patches;                          /* 153 */
  int32_t n_rings;                            /* 8 */
  int32_t bush_any;                           /* bush.max() > 0 */
  int32_t all_finite;                         /* no NaN / inf in dsm, vegdsm, vegdsm2 */
  int32_t step_offset[SW100_MAX_PATCHES];     /* into the step table */
  int32_t step_count[SW100_MAX_PATCHES];
  int32_t ring[SW100_MAX_PATCHES];            /* altitude band of the patch */
  int32_t dir_flags[SW100_MAX_PATCHES];       /* bit0 E, 1 S, 2 W, 3 N */
  int32_t ring_annuli[SW100_MAX_RINGS];       /* annuli per band */
  float w_iso[SW100_MAX_RINGS][SW100_MAX_ANNULI];
  float w_aniso[SW100_MAX_RINGS][SW100_MAX_ANNULI];
  float tail;                                 /* 3.0459e-4 (shadow.py:587) */
  float trans;                                /* 0.03 (shadow.py:612) */
  float trans_veg;                            /* transVeg of the time loop (utci_process.py:864) */
} sw100_svf_plan;

/* out_planes: SW100_SVF_PLANES * npix floats: the reference's 19-tuple
 * order without the cubes, then SVFtotal (svf, svfaveg, svfE, svfEaveg,
 * svfEveg, svfN, svfNaveg, svfNveg, svfS, svfSaveg, svfSveg, svfveg, svfW,
 * svfWaveg, svfWveg, svftotal), then three per-pixel statics of the time
 * loop derived from them: svfbuveg = svf - (1 - svfveg) * (1 - transVeg),
 * tan(acos(sqrt(svf))) and tan(asin(exp(log(1 - tmp) / 2))) with
 * tmp = max(svf + svfveg - 1, 0) (utci_process.py:864-897), each
 * transcendental rounded to float32 once per reference operation.
 * out_bits: 3 cubes (sh, vegsh, vbshvegsh).  plan and steps are device
 * copies of the host tables. */
int sw100_svf_workspace_bytes(int rows, int cols, int n_steps, int64_t* bytes);
int sw100_svf_sweep(const sw100_site_planes* site, int rows, int cols, const sw100_svf_plan* plan,
                    const sw100_step* steps, int n_steps, float* out_planes, uint32_t* out_bits,
                    void* workspace, int64_t workspace_bytes, void* stream);

/* Planes 16-18 of an SVF result (svfbuveg, tan(asvf), tan(svfalfa), as the
 * sweep writes them) from its planes 0 (svf) and 11 (svfveg): for SVF
 * planes that come from elsewhere (the reference's 19-tuple or a cache,
 * utci_process.py:864-897).  planes: SW100_SVF_PLANES * npix floats. */
int sw100_svf_statics(float* planes, int rows, int cols, float trans_veg, void* stream);

/* The same sweep (identical outputs), also counting into *executed (device
 * memory, overwritten) the source gathers its marches execute -- the steps
 * the early exits and the 8-step shortcut leave out are not counted.  Each
 * gather reads the 12 bytes dsm / vegdsm / vegdsm2 that the march step
 * counts of the reference's step tables are defined on
 * (solweig_core/numba_cpu/step_table_gen.py:240-321), so 12 x *executed are
 * the algorithmic bytes of the launch.  For measurement, not for the hot
 * path: the counter costs time. */
int sw100_svf_sweep_count(const sw100_site_planes* site, int rows, int cols, const sw100_svf_plan* plan,
                          const sw100_step* steps, int n_steps, float* out_planes, uint32_t* out_bits,
                          void* workspace, int64_t workspace_bytes, uint64_t* executed, void* stream);

/* ------------------------------------------- windowed SVF recompute -- */
/* Corridor descriptor of one patch for sw100_svf_window (one int32 per
 * patch, built by the host from the step table): bits 0-1 the axis of the
 * patch's major shift (0 = rows / dx, 1 = cols / dy), which is
 * +-(k + 1) at step k, with the minor shift moving by at most one cell per
 * step in one direction; bit 2 set when the major shift is negative.
 * SW100_CORRIDOR_LOCAL marks a patch whose result does not depend on the
 * heights it reads (every step drops the source by more than twice the
 * largest |height|): only pixels inside the edit re-march it.
 * SW100_CORRIDOR_ALWAYS marks a patch whose table has neither form: every
 * window pixel re-marches it. */
#define SW100_CORRIDOR_LOCAL 2
#define SW100_CORRIDOR_ALWAYS 3

/* Exact SVF recompute of a window after an edit of the march rasters.
 *
 * Replaces the corridor-closure work of the reference's incremental exact
 * march (solweig_core/sparse_work.py:633-781 build_sparse_work: per patch,
 * D_p = C u {t : t + d in C} over the executed step offsets d) for one
 * edited rectangle.  `site` holds the edited (post) rasters; `planes` and
 * `bits` hold the sweep result of the rasters before the edit and are
 * updated in place.  rect = {r0, r1, c0, c1} (inclusive) bounds every
 * changed cell; window = {r0, r1, c0, c1} (inclusive, inside the grid) must
 * contain every pixel within the patches' largest shift of the rectangle
 * (pixels outside it cannot reach the rectangle).  Each window pixel
 * re-marches the patches whose march reads the rectangle, keeps the stored
 * bits of the others and re-accumulates its 19 planes in the sweep's
 * order, so the result equals sw100_svf_sweep on the edited rasters bit for
 * bit.  The plan and step tables must be those of the edited rasters and
 * identical to the tables of the stored result (same rows, cols, scale and
 * amaxvalue); rasters with bush (plan bush flag set, before or after the
 * edit) are refused with SW100_E_ARG: their whole-grid step flags change
 * with any edit.  Workspace: sw100_svf_window_workspace_bytes. */
int sw100_svf_window_workspace_bytes(int rows, int cols, int64_t* bytes);
int sw100_svf_window(const sw100_site_planes* site, int rows, int cols, const sw100_svf_plan* plan,
                     const sw100_step* steps, int n_steps, const int32_t* corridor, const int32_t rect[4],
                     const int32_t window[4], float* planes, uint32_t* bits, void* workspace,
                     int64_t workspace_bytes, void* stream);

/* Exact SVF planes and bits of the pixels of a box after an edit inside it,
 * one thread per (pixel, patch) march (low latency for small boxes), then
 * the planes re-accumulated from the bits in the sweep's order.  Pixels
 * outside the box are untouched (their marches may read the box: use
 * sw100_svf_window for an exact update of the whole affected area).  Same
 * tables, corridor descriptors, workspace and refusals as
 * sw100_svf_window.  No counterpart in the reference: it serves the
 * learned preview, which takes the box's own pixels from the exact march. */
int sw100_svf_box(const sw100_site_planes* site, int rows, int cols, const sw100_svf_plan* plan,
                  const sw100_step* steps, int n_steps, const int32_t* corridor, const int32_t box[4], float* planes,
                  uint32_t* bits, void* workspace, int64_t workspace_bytes, void* stream);

/* Bounding box of the cells whose march rasters (dsm, vegdsm, vegdsm2,
 * bush) differ between two sites of the same grid, bit for bit (the
 * composed-source diff C of solweig_core/sparse_work.py:199-251).  Writes
 * {rmin, rmax, cmin, cmax} to the 4 int32 of device memory `box`;
 * rmax = -1 when nothing differs.  Workspace:
 * sw100_diff_bbox_workspace_bytes. */
int sw100_diff_bbox_workspace_bytes(int rows, int cols, int64_t* bytes);
int sw100_diff_bbox(const sw100_site_planes* before, const sw100_site_planes* after, int rows, int cols,
                    int32_t* box, void* workspace, int64_t workspace_bytes, void* stream);

/* Pack dense patch cubes (rows, cols, n_patches) float32, as the reference
 * returns and caches them (shadow.py:625, utci_process.py:347-394), into the
 * 3 bit cubes the time loop reads.  `single_step` (host, SW100_CUBE_WORDS
 * words) marks patches whose SVF march ran at most one step: their
 * vbshvegsh bit records "== 1", every other bit "!= 0". */
int sw100_pack_cubes(const float* shmat, const float* vegshmat, const float* vbshvegshmat, int rows, int cols,
                     int n_patches, const uint32_t* single_step, uint32_t* out_bits, void* stream);

/* SVF sweep that allocates nothing and takes no workspace.
 *
 * This entry point has no counterpart in the reference.  It serves callers
 * that cannot call cudaMalloc themselves: code embedded in a host framework
 * that owns every device allocation through its own pool and forbids direct
 * allocations, or latency-bound loops that cannot afford cudaMalloc /
 * cudaFree (both may synchronise the device).  Such callers still pass
 * their inputs and outputs; the scratch space of the sweep (the packed
 * march source, the bush step flags and the 8 x 8 skip map) lives in a
 * file-scope static device array of SW100_SVF_NOALLOC_SCRATCH_BYTES bytes,
 * which every GPU that loads this library holds until the process exits.
 * The launches are those of sw100_svf_sweep, with that array as the
 * workspace.
 *
 * Limits: the grid must satisfy
 *   sw100_svf_workspace_bytes(rows, cols, n_steps) <= SW100_SVF_NOALLOC_SCRATCH_BYTES
 * i.e. align256(rows * cols * 16) + align256(n_steps * 4)
 *      + align256(ceil(rows / 8) * ceil(cols / 8) * 4)
 * (up to 1024 x 1024 pixels with 65536 table steps); larger requests are
 * refused with SW100_E_SIZE before anything is launched.
 *
 * The first call on each device looks up the array's device address with
 * that device current (cudaGetSymbolAddress) and caches it; make that first
 * call before any stream capture on the device.  The cached address is not
 * refreshed after cudaDeviceReset(): a process that resets a device must not
 * call this entry point on that device again.  All calls share the one
 * array, which keeps the last call's contents (the bush flags are cleared
 * on every call, and the packed source and skip map are rewritten): calls
 * that overlap on the GPU, on different streams or from different threads,
 * race on it and must be serialised by the caller.  Results are identical
 * to sw100_svf_sweep. */
#define SW100_SVF_NOALLOC_SCRATCH_BYTES (16 * 1024 * 1024 + 256 * 1024 + 64 * 1024 + 256)
int sw100_svf_sweep_noalloc(const sw100_site_planes* site, int rows, int cols, const sw100_svf_plan* plan,
                            const sw100_step* steps, int n_steps, float* out_planes, uint32_t* out_bits,
                            void* stream);

/* ------------------------------------------------------ time series -- */
typedef struct {
  int32_t step_offset;     /* into the sun step table */
  int32_t step_count;
  int32_t facesh_mode;     /* 0: az-90 >= 0 and az+90 < 2pi ; 1: wrapped */
  float facesh_lo;         /* float32 thresholds on the wall aspect (rad) */
  float facesh_hi;
  float psi_term;          /* (1 - psi) as float32 */
  int32_t t;               /* time-step index of this daytime row */
  int32_t pad;
} sw100_sun_step;

typedef struct {
  int8_t dx[SW100_MAX_GVF_STEPS];
  int8_t dy[SW100_MAX_GVF_STEPS];
  int32_t facesh_mode;
  float facesh_lo;
  float facesh_hi;
  int32_t dir_flags;        /* bit0 E, 1 S, 2 W, 3 N */
} sw100_gvf_azimuth;

/* per patch and step: increments of the 153-patch sums in the reference's
 * association (solweig.py:683-731 Kside, :1514-1635 define_patch) */
typedef struct {
  float kside_d[4];         /* ((diffsh * lumChi) * anglIncC) * ster; index sh * 2 + vegsh */
  float anilum[4];          /* diffsh * lv */
  /* the rest in 16-byte groups that the loop's set-bit walk reads together */
  float ster;
  float cos_alt;
  float sin_alt;
  float kref_veg;           /* (shaded_surface * ster) * cos(alt) */
  double veg_cos;           /* (vegetation_surface * ster) * cos(alt), float64 */
  double veg_sin;
  float yi_k;               /* yi_ of shaded_or_sunlit, Kside call (float32) */
  float thr_sun;            /* sunlit <=> hsvf + yi < thr_sun */
  float thr_shd;            /* shaded <=> hsvf + yi > thr_shd */
  int32_t flags;            /* bit0: Lcyl sunlit/shaded branch taken */
  float kref_sun;           /* (sunlit_surface * ster) * cos(alt) */
  float kref_sh;            /* (shaded_surface * ster) * cos(alt) */
  float yi_l;               /* yi_ of shaded_or_sunlit, Lcyl call (float32) */
  float ld_sky;             /* Lsky_down[p] */
  float sun_cos;            /* (sunlit wall surface * ster) * cos(alt) */
  float sun_sin;
  float ls_sky;             /* Lsky_side[p] */
  int32_t pad;
  double sh_cos;            /* (shaded_surface * ster) * cos(alt), float64 */
  double sh_sin;
} sw100_patch_step;

typedef struct {
  int32_t is_day;
  int32_t day_row;          /* row of this step in the sun-march output, -1 at night */
  int32_t tw_mode;          /* TsWaveDelay: 1 -> Tgmap1 updated, 0 -> lag only */
  int32_t tw_first;         /* firstdaytime == 1 at this step */
  float tw_a;               /* (1 - weight1) */
  float tw_b;               /* weight1 */
  float ta32;               /* Ta as float32 */
  float ta4;                /* (Ta + 273.15) ** 4 as float32 */
  float sbc;                /* 5.67051e-8 as float32 */
  float altmax32;
  float cig;                /* CI_TgG as float32 */
  float lwall;              /* Lwall of sunonsurface_2018a */
  float radI, radD, radG;   /* float32 */
  float sin_alt;            /* float32(sin(altitude)) for Kdown / Kup */
  float cos_alt;            /* float32(cos(altitude)) for KsideI */
  float albedo_b;
  float first, second;      /* ground-view-factor walk lengths (rounded) */
  float tan_beta;           /* tan(zen) float32 for cylindric_wedge */
  float qa;                 /* tan(beta) / 2 */
  float refl_k;             /* (1 - ewall) as float32 */
  float night_lup_base;     /* night: float32 (0 + Ta) + 0 + 273.15 */
  float absK, absL, Fside, Fup, Fcyl;
  float absl_sbc;           /* absL * SBC (float32) */
  float rh32;               /* RH for UTCI */
  float ws32;               /* wind speed */
  float ta_mat;             /* float32(Ta) + float32(uhii) */
  int32_t landcover;        /* Tg = max(Tg, 0) when land cover is used */
  float tg_factor[SW100_MAX_CLASSES]; /* sin(...) of the Tg wave per TmaxLST class */
  /* UTCI of this step (calculate_utci.py:259-330, float32 as the reference
   * evaluates it): Pa^1..Pa^6 of this step's vapour pressure, and per
   * regression term j the float32 product c_j * Ta^pt_j (c_j when pt_j == 0);
   * the kernel multiplies in va, D = Tmrt - Ta and Pa and sums in order */
  float utci_pa[6];
  float utci_k[SW100_UTCI_TERMS];
  int32_t pad1[2];
} sw100_time_step;

/* All tables of one site's time loop (device pointers). */
typedef struct {
  const sw100_time_step* steps;     /* n_t */
  int32_t n_t;
  int32_t n_day;
  const sw100_sun_step* sun;        /* n_day */
  const sw100_step* sun_table;      /* concatenated sun-march step tables */
  const sw100_patch_step* patch;    /* n_t * n_patches */
  int32_t n_patches;
  int32_t pad;
  const sw100_gvf_azimuth* gvf;     /* SW100_N_GVF_AZ */
} sw100_series;

/* Output selection bits for sw100_time_loop (reference variable names). */
#define SW100_OUT_UTCI   (1 << 0)
#define SW100_OUT_TMRT   (1 << 1)
#define SW100_OUT_KUP    (1 << 2)
#define SW100_OUT_KDOWN  (1 << 3)
#define SW100_OUT_LUP    (1 << 4)
#define SW100_OUT_LDOWN  (1 << 5)
#define SW100_OUT_SHADOW (1 << 6)

/* ------------------------------------------------------------ batches -- */
/* One site of a batched launch.  A device array of these, and device tile
 * lists, drive the sw100_batch_* entry points: every stage of every site of
 * the batch runs in one launch per stage (the reference runs one site at a
 * time, utci_process.py:1472-1651 run_utci_tiles / solweig_gpu.py:387-497).
 * All pointers are device memory.  `site.bits`, `site.svfbuveg`,
 * `site.hsvf` and `site.tan_alfa` point into `svf_bits` / `svf_planes`
 * (planes 16, 17, 18), `site.single_step` holds the SVF plan's one-step
 * patches, so the time loop reads what the sweep of the same batch wrote. */
typedef struct {
  sw100_site_planes site;
  int32_t rows, cols;
  const sw100_svf_plan* plan;   /* SVF tables of the site (sw100_svf_sweep) */
  const sw100_step* steps;
  sw100_series series;          /* time-series tables of the site (sw100_time_loop) */
  float* svf_planes;            /* SW100_SVF_PLANES * npix, written by the sweep */
  uint32_t* svf_bits;           /* 3 * SW100_CUBE_WORDS * npix, written by the sweep */
  float* src4;                  /* 4 * npix, packed march source */
  uint32_t* bflags;             /* one word per SVF table step, zeroed by the caller (bush sites) */
  float* gsrc;                  /* 4 * n_day * npix, sun-march records */
  float* state;                 /* 6 * npix thermal state, carried across calls */
  float* outputs;               /* popcount(out_mask) * n_t * npix */
  uint32_t out_mask;
  int32_t svf_steps;            /* entries of the step table `steps` */
  float* skipmap;               /* ((rows + 7) / 8) * ((cols + 7) / 8) source bounds of the SVF
                                   sweep, written by sw100_batch_skipmap after the pack; NULL:
                                   march every step */
  const float* sums;            /* n_t * 4 * npix dense patch sums of the site's series, written by
                                   sw100_patch_sums after the sweep; read by
                                   sw100_batch_flux_loop_sums (NULL for sw100_batch_flux_loop) */
} sw100_batch_site;

/* Tile list entry {site index, tile column, tile row, daytime row}: the
 * tile covers pixels [tile column * block_x, +block_x) x [tile row *
 * block_y, +block_y) of its site; the daytime row is used by the sun march
 * only.  Lists are ordered by the caller (heaviest sites first). */
typedef struct {
  int32_t site, tx, ty, day;
} sw100_tile;

/* Checks a host copy of the batch descriptors (sizes, pointers, patch
 * counts) before the caller uploads it. */
int sw100_batch_validate(const sw100_batch_site* host_sites, int n_sites);
/* Each launch runs `grid` blocks of block_x * block_y == 128 threads over
 * the tile list (grid < n_tiles: blocks stride over the list, a persistent
 * launch; grid == n_tiles: one tile per block).  Stages: pack the march
 * sources; the bush step flags of bush sites (tiles of those sites only);
 * the SVF sweep; the sun march (tiles carry the daytime row); the flux
 * loop. */
int sw100_batch_pack(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x,
                     int block_y, int grid, void* stream);
int sw100_batch_bush_flags(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x,
                           int block_y, int grid, void* stream);
/* Source-height bounds of 8 x 8 cell blocks (the step shortcut of the SVF
 * sweep) for every site of `sites` (device array of n_sites) whose skipmap
 * is not NULL; runs after the pack. */
int sw100_batch_skipmap(const sw100_batch_site* sites, int n_sites, void* stream);
int sw100_batch_svf(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x, int block_y,
                    int grid, void* stream);
int sw100_batch_sun_march(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x,
                          int block_y, int grid, void* stream);
int sw100_batch_flux_loop(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x,
                          int block_y, int grid, void* stream);
/* sw100_batch_flux_loop with every site's dense patch sums read from its
 * `sums` (sw100_flux_loop_sums per site: fluxes held to the Tmrt / UTCI
 * tolerance); every listed site must have `sums` set. */
int sw100_batch_flux_loop_sums(const sw100_batch_site* sites, const sw100_tile* tiles, int n_tiles, int block_x,
                               int block_y, int grid, void* stream);

/* Sun march for every daytime row of the series in one launch.  Writes the
 * per-row ground-view-factor source records (4 floats per pixel:
 * shadow, Lup, albedo, flag bits) to gsrc (n_day * npix * 4 floats) and,
 * when debug8 is non-NULL, the 8 planes of the reference return tuple
 * (vegsh, sh, vbshvegsh, wallsh, wallsun, wallshve, facesh, facesun) at
 * debug8[(d * 8 + k) * npix]. */
int sw100_sun_march_workspace_bytes(int rows, int cols, int64_t* bytes);
int sw100_sun_march(const sw100_site_planes* site, int rows, int cols, const sw100_series* series,
                    float* gsrc, float* debug8, void* workspace, int64_t workspace_bytes, void* stream);

/* All steps of one site's time loop: sun march of the daytime rows, then
 * one launch for ground view factors, thermal lag (state carried in
 * registers), K/L fluxes, Tmrt and UTCI.  `state` holds the 6 thermal planes
 * (Tgmap1, E, S, W, N, TgOut1), read at the start and written at the end.
 * `outputs` receives, for each bit set in `out_mask` (in bit order), an
 * n_t * npix block. */
int sw100_time_loop_workspace_bytes(int rows, int cols, int n_day, int64_t* bytes);
int sw100_time_loop(const sw100_site_planes* site, int rows, int cols, const sw100_series* series,
                    float* state, uint32_t out_mask, float* outputs, void* workspace,
                    int64_t workspace_bytes, void* stream);

/* The fused loop kernel of sw100_time_loop alone, reading sun-march records
 * from a previous sw100_sun_march call on the same series (gsrc as written
 * there, n_day * npix * 4 floats).  Lets a caller time or overlap the two
 * launches separately; no workspace. */
int sw100_flux_loop(const sw100_site_planes* site, int rows, int cols, const sw100_series* series,
                    const float* gsrc, float* state, uint32_t out_mask, float* outputs, void* stream);

/* The dense 153-patch sums of the time loop on the tensor cores
 * (solweig.py:683-724 diffuse Kside and anisotropic luminance,
 * :1514-1541 sky longwave): for every step t of the series and pixel p,
 *   sums[(t * 4 + 0) * npix + p] = diffuse Kside (0 at night),
 *   sums[(t * 4 + 1) * npix + p] = anisotropic luminance sum (0 at night),
 *   sums[(t * 4 + 2) * npix + p] = sky longwave down,
 *   sums[(t * 4 + 3) * npix + p] = sky longwave side,
 * as a product of the pixel's one-hot (sh, vegsh) patch codes (from
 * site->bits) with the series' per-patch increments, each split into three
 * bf16 parts that add up to the float32 increment; FP32 accumulation
 * (tcgen05.mma, accumulator in tensor memory).  The sums equal the
 * reference's patch-ordered float32 sums to about one rounding.
 * `err` (device int32, may be NULL) is set to 1 when a bounded wait of the
 * kernel expired (then the block writes nothing), 2 when its drain did too.
 * Workspace: sw100_patch_sums_workspace_bytes (the bf16 weights). */
int sw100_patch_sums_workspace_bytes(int n_t, int64_t* bytes);
int sw100_patch_sums(const sw100_site_planes* site, int rows, int cols, const sw100_series* series, float* sums,
                     int32_t* err, void* workspace, int64_t workspace_bytes, void* stream);

/* Ground-view walk work of each 8 x 4 pixel patch of the time / flux loops
 * (patch numbering of sw100_site_planes.patch_order): for each of the 18
 * azimuths of `gvf` (sw100_gvf_azimuth rows of the loops' series) the
 * longest walk of the patch's pixels up to the first building sample
 * (site->buildings == 0, in the grid) or `second` steps, summed over the
 * azimuths.  `work` holds ceil(rows / 4) * ceil(cols / 8) int32.  No
 * reference counterpart: a scheduling input. */
int sw100_walk_work(const sw100_site_planes* site, int rows, int cols, const sw100_gvf_azimuth* gvf, int second,
                    int32_t* work, void* stream);

/* sw100_flux_loop with the dense patch sums taken from `sums` (as written
 * by sw100_patch_sums for the same series) instead of computed in the
 * loop.  Its fluxes are held to the Tmrt / UTCI tolerance of the chain
 * (1e-3 K / 1e-3 C against the reference) rather than to the reference's
 * float32 operation order: besides the tensor-core sums, the vegetation and
 * shaded-wall longwave sums stay in float64 to the end, the reflected
 * longwave is refl x sum(ster x cos) by FMA, and the ground-view weights
 * divide by multiplying with the step's reciprocals.  Shadows and every
 * predicate (sunlit / shaded walls, the first-building walks) are the
 * reference's. */
int sw100_flux_loop_sums(const sw100_site_planes* site, int rows, int cols, const sw100_series* series,
                         const float* gsrc, const float* sums, float* state, uint32_t out_mask, float* outputs,
                         void* stream);

/* ---------------------------------------------------- learned preview -- */
/* Kernels of the learned SVF preview (a small U-Net, BF16 on the tensor
 * cores with FP32 accumulation).  No counterpart in the reference: the
 * reference recomputes SVF exactly for every edit (shadow.py:409-625 /
 * solweig_core/sparse_work.py); the preview is a fast approximate edit path
 * whose error is checked, and which is replaced when too large, by the exact
 * windowed recompute (sw100_svf_window).
 *
 * Activations are NHWC bf16; a layer reads / writes channels [coff, coff +
 * C) of a buffer of `stride` channels (C, coff, stride multiples of 16).
 * 3 x 3 convolutions use same padding and tap t = 3 (dy + 1) + (dx + 1);
 * weights: forward layout [t][cout][cin] bf16, data-gradient layout
 * [8 - t][cin][cout] bf16, float32 master weights / gradients in the
 * forward layout. */
/* y[., ycoff + co] = act(bias[co] + sum_{t, ci} x[shifted, xcoff + ci] *
 * wt[t][co][ci]) on the 5th-generation tensor cores (tcgen05.mma with the
 * accumulator in tensor memory; cout <= 128); relu: max(0, .), out_f32:
 * float32 output instead of bf16, bias may be NULL.  A data gradient is
 * this call on the output gradient with the data-gradient weight layout.
 * err (device int32, may be NULL) is set to 1 when a bounded wait of the
 * kernel expired: the block then issues no further copy or MMA, waits for
 * the MMAs it issued (with the default limit), frees its tensor memory and
 * writes no output; err is set to 2 when that drain ran out as well. */
int sw100_nn_conv3x3_tc(const void* x, int n, int h, int w, int cin, int xstride, int xcoff, const void* wt,
                        const float* bias, int cout, void* y, int ystride, int ycoff, int relu, int out_f32,
                        int32_t* err, void* stream);
/* Polls of an mbarrier before a wait of the tensor-core kernels gives up
 * (default 2^22; a negative value restores it).  Returns the previous
 * limit.  Process-wide; meant for tests of the timeout path (a limit of 0
 * makes every pipeline wait run out at once).  No counterpart in the
 * reference. */
int sw100_set_wait_limit(int polls);
/* dw (float32, forward layout) and dbias (may be NULL) += the gradients of
 * a 3 x 3 convolution given its input x and output gradient dy. */
int sw100_nn_conv3x3_wgrad(const void* x, int n, int h, int w, int cin, int xstride, int xcoff, const void* dy,
                           int cout, int dstride, int dcoff, float* dw, float* dbias, void* stream);
/* float32 master weights -> bf16 forward layout wf and data-gradient layout wd (may be NULL). */
int sw100_nn_weights(const float* master, int cin, int cout, void* wf, void* wd, void* stream);
/* dy *= (y > 0) (ReLU backward on the layer's output y). */
int sw100_nn_relu_bwd(void* dy, const void* y, int64_t npix, int c, int dstride, int dcoff, int ystride, int ycoff,
                      void* stream);
/* 2 x 2 average pooling (h, w: input size) and its backward (x = dY of
 * size h/2 x w/2, y = dX, accumulate: add into dX). */
int sw100_nn_pool2(const void* x, int n, int h, int w, int c, int xstride, int xcoff, void* y, int ystride, int ycoff,
                   int backward, int accumulate, void* stream);
/* nearest 2x upsampling (h, w: input size) and its backward (x = dY of
 * size 2h x 2w, y = dX). */
int sw100_nn_up2(const void* x, int n, int h, int w, int c, int xstride, int xcoff, void* y, int ystride, int ycoff,
                 int backward, void* stream);
/* mean squared error over the central box (margin cells cut on each side)
 * and the first nc of c channels of float32 NHWC pred / target; loss
 * (float32, may be NULL) += the mean, dpred (bf16, may be NULL) = its
 * gradient. */
int sw100_nn_mse(const float* pred, const float* target, int n, int h, int w, int c, int nc, int margin, void* dpred,
                 float* loss, void* stream);
/* One bias-corrected Adam step (Kingma & Ba 2015) on float32 parameters. */
int sw100_nn_adam(float* param, const float* grad, float* m, float* v, int64_t n, float lr, float b1, float b2,
                  float eps, int step, void* stream);
/* Network input of n square windows of `size` cells at device origins
 * {r0, c0} (int32 pairs) of a site: heights above ground of the building
 * DSM, canopy top and trunk zone, / 40 m, bf16 NHWC with 16 channels (3
 * used); cells outside the grid read 0.  dem may be NULL (flat 0). */
int sw100_nn_input(const float* dsm, const float* vegdsm, const float* vegdsm2, const float* dem, int rows, int cols,
                   const int32_t* origins, int n, int size, void* x, void* stream);

/* ---------------------------------------------------------------- UTCI -- */
/* UTCI-only recompute of whole steps: the met fast path of
 * utci_process.py:1093-1196 (recompute_utci_steps), for wind speed / urban
 * heat island edits that leave Tmrt unchanged.  steps: n_steps records whose
 * ta_mat, rh32, ws32, utci_pa and utci_k are set (the other fields are not
 * read); tmrt: n_steps * npix stored Tmrt planes; buildings: 1 where UTCI
 * is defined (NaN elsewhere); windcoeff: npix or NULL (1).  out: n_steps *
 * npix.  The arithmetic is the time loop's UTCI tail, so the result equals
 * the UTCI a full run would give for the same forcing and Tmrt. */
int sw100_utci_steps(const sw100_time_step* steps, int n_steps, const float* tmrt, const float* buildings,
                     const float* windcoeff, int64_t npix, float* out, void* stream);

/* utci_calculator over n float32 elements: saturation vapour pressure from
 * Ta, then the 210-term regression in float64; -999 where any input is
 * <= -999 (calculate_utci.py:259-330). */
int sw100_utci(const float* ta, const float* rh, const float* tmrt, const float* va, int64_t n,
               float* out, void* stream);

/* ------------------------------------------------------------ support -- */
int sw100_abi_version(void);
const char* sw100_last_error(void);
/* number of kernels this library has launched since it was loaded */
int64_t sw100_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* SOLWEIG_B200_H */
