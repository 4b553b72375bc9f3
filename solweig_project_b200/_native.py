"""ctypes binding of ``libsolweig_b200.so`` (the C ABI in include/solweig_b200.h).

The library is built in-tree by :mod:`solweig_project_b200.build`.  Loading
never falls back to anything: a missing or stale library raises
:class:`NativeUnavailable`, and every non-zero status from the library raises
:class:`NativeError` carrying ``sw100_last_error()``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libsolweig_b200.so")

CUBE_WORDS = 5
MAX_PATCHES = 160
MAX_RINGS = 16
MAX_ANNULI = 16
MAX_CLASSES = 8
N_GVF_AZ = 18
UTCI_TERMS = 210
MAX_GVF_STEPS = 64
SVF_PLANES = 19
SVF_NOALLOC_SCRATCH_BYTES = 16 * 1024 * 1024 + 256 * 1024 + 64 * 1024 + 256

OUT_UTCI, OUT_TMRT, OUT_KUP, OUT_KDOWN, OUT_LUP, OUT_LDOWN, OUT_SHADOW = (1 << i for i in range(7))
OUT_BITS = {"utci": OUT_UTCI, "tmrt": OUT_TMRT, "kup": OUT_KUP, "kdown": OUT_KDOWN, "lup": OUT_LUP,
            "ldown": OUT_LDOWN, "shadow": OUT_SHADOW}

# Exported symbols (checked by the CPU tests against include/solweig_b200.h)
SYMBOLS = ("sw100_svf_workspace_bytes", "sw100_svf_sweep", "sw100_svf_sweep_count", "sw100_svf_statics", "sw100_svf_sweep_noalloc", "sw100_pack_cubes",
           "sw100_sun_march_workspace_bytes", "sw100_sun_march", "sw100_time_loop_workspace_bytes", "sw100_time_loop",
           "sw100_flux_loop", "sw100_utci", "sw100_abi_version", "sw100_last_error", "sw100_launch_count",
           "sw100_svf_window_workspace_bytes", "sw100_svf_window", "sw100_diff_bbox_workspace_bytes",
           "sw100_diff_bbox", "sw100_batch_validate", "sw100_batch_pack", "sw100_batch_bush_flags",
           "sw100_batch_skipmap", "sw100_batch_svf", "sw100_batch_sun_march", "sw100_batch_flux_loop",
           "sw100_batch_flux_loop_sums", "sw100_utci_steps", "sw100_nn_conv3x3_wgrad", "sw100_nn_weights",
           "sw100_nn_relu_bwd", "sw100_nn_pool2",
           "sw100_nn_up2", "sw100_nn_mse", "sw100_nn_adam", "sw100_nn_input", "sw100_svf_box", "sw100_nn_conv3x3_tc",
           "sw100_prepare_site", "sw100_march_tables", "sw100_set_wait_limit",
           "sw100_patch_sums_workspace_bytes", "sw100_patch_sums", "sw100_flux_loop_sums", "sw100_walk_work")
ABI_VERSION = 3  # SW100_ABI_VERSION of include/solweig_b200.h
CORRIDOR_LOCAL = 2
CORRIDOR_ALWAYS = 3


class NativeUnavailable(RuntimeError):
    """The CUDA library is missing or could not be loaded."""


class NativeError(RuntimeError):
    """A library entry point returned a non-zero status."""

    def __init__(self, fn, code, message):
        super().__init__(f"{fn} failed with status {code}: {message}")
        self.code = code
        self.message = message


# ----------------------------------------------------------- numpy tables
STEP_DTYPE = np.dtype([("dx", "<i4"), ("dy", "<i4"), ("dz", "<f4"), ("flags", "<i4")], align=True)
MARCH_CONST_DTYPE = np.dtype([("branch_y", "<i4"), ("ssin", "<f4"), ("scos", "<f4"), ("tan_a", "<f4"),
                              ("ds", "<f4"), ("tanalt", "<f4")], align=True)
STEP_SKIP8 = 1

SVF_PLAN_DTYPE = np.dtype([
    ("n_patches", "<i4"), ("n_rings", "<i4"), ("bush_any", "<i4"), ("all_finite", "<i4"),
    ("step_offset", "<i4", (MAX_PATCHES,)), ("step_count", "<i4", (MAX_PATCHES,)),
    ("ring", "<i4", (MAX_PATCHES,)), ("dir_flags", "<i4", (MAX_PATCHES,)),
    ("ring_annuli", "<i4", (MAX_RINGS,)),
    ("w_iso", "<f4", (MAX_RINGS, MAX_ANNULI)), ("w_aniso", "<f4", (MAX_RINGS, MAX_ANNULI)),
    ("tail", "<f4"), ("trans", "<f4"), ("trans_veg", "<f4"),
], align=True)

SUN_STEP_DTYPE = np.dtype([
    ("step_offset", "<i4"), ("step_count", "<i4"), ("facesh_mode", "<i4"), ("facesh_lo", "<f4"),
    ("facesh_hi", "<f4"), ("psi_term", "<f4"), ("t", "<i4"), ("pad", "<i4"),
], align=True)

GVF_AZ_DTYPE = np.dtype([
    ("dx", "i1", (MAX_GVF_STEPS,)), ("dy", "i1", (MAX_GVF_STEPS,)), ("facesh_mode", "<i4"),
    ("facesh_lo", "<f4"), ("facesh_hi", "<f4"), ("dir_flags", "<i4"),
], align=True)

PATCH_STEP_DTYPE = np.dtype([
    ("kside_d", "<f4", (4,)), ("anilum", "<f4", (4,)),
    ("ster", "<f4"), ("cos_alt", "<f4"), ("sin_alt", "<f4"), ("kref_veg", "<f4"),
    ("veg_cos", "<f8"), ("veg_sin", "<f8"),
    ("yi_k", "<f4"), ("thr_sun", "<f4"), ("thr_shd", "<f4"), ("flags", "<i4"),
    ("kref_sun", "<f4"), ("kref_sh", "<f4"), ("yi_l", "<f4"), ("ld_sky", "<f4"),
    ("sun_cos", "<f4"), ("sun_sin", "<f4"), ("ls_sky", "<f4"), ("pad", "<i4"),
    ("sh_cos", "<f8"), ("sh_sin", "<f8"),
], align=True)

TIME_STEP_DTYPE = np.dtype([
    ("is_day", "<i4"), ("day_row", "<i4"), ("tw_mode", "<i4"), ("tw_first", "<i4"),
    ("tw_a", "<f4"), ("tw_b", "<f4"), ("ta32", "<f4"), ("ta4", "<f4"), ("sbc", "<f4"),
    ("altmax32", "<f4"), ("cig", "<f4"), ("lwall", "<f4"), ("radI", "<f4"), ("radD", "<f4"),
    ("radG", "<f4"), ("sin_alt", "<f4"), ("cos_alt", "<f4"), ("albedo_b", "<f4"), ("first", "<f4"),
    ("second", "<f4"), ("tan_beta", "<f4"), ("qa", "<f4"), ("refl_k", "<f4"), ("night_lup_base", "<f4"),
    ("absK", "<f4"), ("absL", "<f4"), ("Fside", "<f4"), ("Fup", "<f4"), ("Fcyl", "<f4"),
    ("absl_sbc", "<f4"), ("rh32", "<f4"), ("ws32", "<f4"), ("ta_mat", "<f4"), ("landcover", "<i4"),
    ("tg_factor", "<f4", (MAX_CLASSES,)), ("utci_pa", "<f4", (6,)), ("utci_k", "<f4", (UTCI_TERMS,)),
    ("pad1", "<i4", (2,)),
], align=True)

EXPECTED_SIZES = {"sw100_step": 16, "sw100_svf_plan": 4700, "sw100_sun_step": 32,
                  "sw100_gvf_azimuth": 144, "sw100_patch_step": 128, "sw100_time_step": 1040}
DTYPES = {"sw100_step": STEP_DTYPE, "sw100_svf_plan": SVF_PLAN_DTYPE, "sw100_sun_step": SUN_STEP_DTYPE,
          "sw100_gvf_azimuth": GVF_AZ_DTYPE, "sw100_patch_step": PATCH_STEP_DTYPE,
          "sw100_time_step": TIME_STEP_DTYPE}


# ------------------------------------------------------- ctypes structures
class SitePlanes(C.Structure):
    _fields_ = [
        ("dsm", C.c_void_p), ("vegdsm", C.c_void_p), ("vegdsm2", C.c_void_p), ("bush", C.c_void_p),
        ("vmax", C.c_float), ("bush_any", C.c_int32),
        ("svfbuveg", C.c_void_p), ("hsvf", C.c_void_p), ("tan_alfa", C.c_void_p), ("buildings", C.c_void_p),
        ("walls", C.c_void_p), ("aspect_rad", C.c_void_p), ("tgk", C.c_void_p), ("tstart", C.c_void_p),
        ("alb", C.c_void_p), ("emis", C.c_void_p), ("class_idx", C.c_void_p), ("windcoeff", C.c_void_p),
        ("bits", C.c_void_p), ("single_step", C.c_uint32 * CUBE_WORDS),
        ("patch_order", C.c_void_p), ("n_patch_order", C.c_int32),
    ]


class ClassTable(C.Structure):
    """sw100_class_table: land-cover properties by cleaned code."""
    _fields_ = [("tgk", C.c_float * 8), ("tstart", C.c_float * 8), ("alb", C.c_float * 8), ("emis", C.c_float * 8),
                ("valid", C.c_uint32)]


N_SITE_STATS = 8
STAT_DSM, STAT_VEGDEM, STAT_VEGDSM, STAT_VEGDSM2, STAT_ABS_DSM, STAT_ABS_VEGDSM, STAT_ABS_VEGDSM2, STAT_BUSH = range(8)
SITE_STATS_WORDS = N_SITE_STATS + 4   # sw100_site_stats as uint32 words


def stat_value(stats: np.ndarray, s: int) -> np.float32:
    """Maximum s of a sw100_site_stats read back as uint32 words: NaN when a
    NaN entered it, else the float whose order-preserving key is stored."""
    if (int(stats[N_SITE_STATS]) >> s) & 1:
        return np.float32(np.nan)
    k = int(stats[s])
    u = (k & 0x7fffffff) if k & 0x80000000 else (~k & 0xffffffff)
    return np.array([u], np.uint32).view(np.float32)[0]


class Series(C.Structure):
    _fields_ = [
        ("steps", C.c_void_p), ("n_t", C.c_int32), ("n_day", C.c_int32), ("sun", C.c_void_p),
        ("sun_table", C.c_void_p), ("patch", C.c_void_p), ("n_patches", C.c_int32), ("pad", C.c_int32),
        ("gvf", C.c_void_p),
    ]


_LIB = None


def load(path: str = LIB_PATH):
    """Load the library once (raises :class:`NativeUnavailable`)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise NativeUnavailable(f"{path} is missing; build it with `python -m solweig_project_b200.build`")
    try:
        lib = C.CDLL(path)
    except OSError as exc:  # pragma: no cover - depends on the loader
        raise NativeUnavailable(f"cannot load {path}: {exc}") from exc
    i64p = C.POINTER(C.c_int64)
    vp = C.c_void_p
    sig = {
        "sw100_abi_version": (C.c_int, []),
        "sw100_last_error": (C.c_char_p, []),
        "sw100_launch_count": (C.c_int64, []),
        "sw100_svf_workspace_bytes": (C.c_int, [C.c_int, C.c_int, C.c_int, i64p]),
        "sw100_svf_sweep": (C.c_int, [C.POINTER(SitePlanes), C.c_int, C.c_int, vp, vp, C.c_int, vp, vp, vp,
                                      C.c_int64, vp]),
        "sw100_svf_sweep_count": (C.c_int, [C.POINTER(SitePlanes), C.c_int, C.c_int, vp, vp, C.c_int, vp, vp, vp,
                                            C.c_int64, vp, vp]),
        "sw100_svf_statics": (C.c_int, [vp, C.c_int, C.c_int, C.c_float, vp]),
        "sw100_svf_sweep_noalloc": (C.c_int, [C.POINTER(SitePlanes), C.c_int, C.c_int, vp, vp, C.c_int, vp, vp,
                                              vp]),
        "sw100_pack_cubes": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint32), vp, vp]),
        "sw100_sun_march_workspace_bytes": (C.c_int, [C.c_int, C.c_int, i64p]),
        "sw100_sun_march": (C.c_int, [C.POINTER(SitePlanes), C.c_int, C.c_int, C.POINTER(Series), vp, vp, vp,
                                      C.c_int64, vp]),
        "sw100_time_loop_workspace_bytes": (C.c_int, [C.c_int, C.c_int, C.c_int, i64p]),
        "sw100_time_loop": (C.c_int, [C.POINTER(SitePlanes), C.c_int, C.c_int, C.POINTER(Series), vp, C.c_uint32,
                                      vp, vp, C.c_int64, vp]),
        "sw100_flux_loop": (C.c_int, [C.POINTER(SitePlanes), C.c_int, C.c_int, C.POINTER(Series), vp, vp, C.c_uint32,
                                      vp, vp]),
        "sw100_patch_sums_workspace_bytes": (C.c_int, [C.c_int, i64p]),
        "sw100_patch_sums": (C.c_int, [C.POINTER(SitePlanes), C.c_int, C.c_int, C.POINTER(Series), vp, vp, vp,
                                       C.c_int64, vp]),
        "sw100_walk_work": (C.c_int, [C.POINTER(SitePlanes), C.c_int, C.c_int, vp, C.c_int, vp, vp]),
        "sw100_flux_loop_sums": (C.c_int, [C.POINTER(SitePlanes), C.c_int, C.c_int, C.POINTER(Series), vp, vp, vp,
                                           C.c_uint32, vp, vp]),
        "sw100_utci": (C.c_int, [vp, vp, vp, vp, C.c_int64, vp, vp]),
        "sw100_svf_window_workspace_bytes": (C.c_int, [C.c_int, C.c_int, i64p]),
        "sw100_svf_window": (C.c_int, [C.POINTER(SitePlanes), C.c_int, C.c_int, vp, vp, C.c_int, vp,
                                       C.POINTER(C.c_int32), C.POINTER(C.c_int32), vp, vp, vp, C.c_int64, vp]),
        "sw100_diff_bbox_workspace_bytes": (C.c_int, [C.c_int, C.c_int, i64p]),
        "sw100_svf_box": (C.c_int, [C.POINTER(SitePlanes), C.c_int, C.c_int, vp, vp, C.c_int, vp, C.POINTER(C.c_int32),
                                    vp, vp, vp, C.c_int64, vp]),
        "sw100_batch_validate": (C.c_int, [vp, C.c_int]),
        "sw100_utci_steps": (C.c_int, [vp, C.c_int, vp, vp, vp, C.c_int64, vp, vp]),
        "sw100_nn_conv3x3_tc": (C.c_int, [vp] + [C.c_int] * 6 + [vp, vp, C.c_int, vp] + [C.c_int] * 4 + [vp, vp]),
        "sw100_nn_conv3x3_wgrad": (C.c_int, [vp] + [C.c_int] * 6 + [vp] + [C.c_int] * 3 + [vp, vp, vp]),
        "sw100_nn_weights": (C.c_int, [vp, C.c_int, C.c_int, vp, vp, vp]),
        "sw100_nn_relu_bwd": (C.c_int, [vp, vp, C.c_int64] + [C.c_int] * 5 + [vp]),
        "sw100_nn_pool2": (C.c_int, [vp] + [C.c_int] * 6 + [vp] + [C.c_int] * 4 + [vp]),
        "sw100_nn_up2": (C.c_int, [vp] + [C.c_int] * 6 + [vp] + [C.c_int] * 3 + [vp]),
        "sw100_nn_mse": (C.c_int, [vp, vp] + [C.c_int] * 6 + [vp, vp, vp]),
        "sw100_nn_adam": (C.c_int, [vp, vp, vp, vp, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                    vp]),
        "sw100_nn_input": (C.c_int, [vp, vp, vp, vp, C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, vp]),
        **{name: (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp]) for name in (
            "sw100_batch_pack", "sw100_batch_bush_flags", "sw100_batch_svf", "sw100_batch_sun_march",
            "sw100_batch_flux_loop", "sw100_batch_flux_loop_sums")},
        "sw100_batch_skipmap": (C.c_int, [vp, C.c_int, vp]),
        "sw100_set_wait_limit": (C.c_int, [C.c_int]),
        "sw100_prepare_site": (C.c_int, [vp, vp, vp, vp, vp, C.POINTER(ClassTable), C.c_int, C.c_int] + [vp] * 12),
        "sw100_march_tables": (C.c_int, [vp, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, vp, C.c_int64, vp,
                                         i64p]),
        "sw100_diff_bbox": (C.c_int, [C.POINTER(SitePlanes), C.POINTER(SitePlanes), C.c_int, C.c_int, vp, vp,
                                      C.c_int64, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.sw100_abi_version() != ABI_VERSION:
        raise NativeUnavailable(f"{path} has ABI version {lib.sw100_abi_version()}, expected {ABI_VERSION}")
    _LIB = lib
    return lib


def call(name: str, *args) -> None:
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != 0:
        msg = lib.sw100_last_error()
        raise NativeError(name, rc, msg.decode() if msg else "")


def workspace_bytes(name: str, *args) -> int:
    out = C.c_int64(0)
    call(name, *args, C.byref(out))
    return int(out.value)


def launch_count() -> int:
    return int(load().sw100_launch_count())


def march_tables(consts: np.ndarray, first_index: int, amax, rows: int, cols: int):
    """sw100_march_tables: (steps, counts) of the marches described by the
    MARCH_CONST_DTYPE records `consts` (host arrays; no device work)."""
    consts = np.ascontiguousarray(consts, MARCH_CONST_DTYPE)
    n = len(consts)
    counts = np.zeros(max(n, 1), np.int32)
    total = C.c_int64(0)
    cp = consts.ctypes.data if n else None
    # room for every march at its longest (max(rows, cols) + 3 - first_index
    # steps): one call that counts and fills in one pass
    cap = n * max(0, max(int(rows), int(cols)) + 3 - int(first_index))
    buf = np.empty(max(cap, 1), STEP_DTYPE)
    call("sw100_march_tables", cp, n, int(first_index), C.c_float(np.float32(amax)), int(rows), int(cols),
         buf.ctypes.data, cap, counts.ctypes.data, C.byref(total))
    return buf[:int(total.value)], counts[:n].astype(np.int64)
