"""Host-side march and patch tables for the CUDA kernels.

The kernels consume precomputed tables instead of re-deriving the scalar
geometry on the device: the reference evaluates that geometry with 0-dim
float32 torch tensors (sin/cos/tan of the march azimuth, tan of the altitude,
the branch bounds) and the exact float32 bits decide which pixels are shadowed.
Here the transcendental calls go through the same torch CPU kernels and the
remaining per-step arithmetic (round-half-even, products, the while-loop stop
rule) is IEEE float32 in numpy, vectorised over the steps.

* SVF patch layout and weights: ``solweig_gpu/shadow.py:324-406, 530-543``
* SVF patch march tables: ``shadow.py:196-247`` (index from 1, azimuth 0
  replaced by 1e-12, python-float branch bounds)
* sun march tables: ``solweig_gpu/solweig.py:1092-1149`` (index from 0,
  float32 tensor branch bounds)
* ground-view-factor walk offsets: ``solweig.py:136-178``
"""
from __future__ import annotations

import functools

import numpy as np
import torch

from . import _native as N

F32 = np.float32

# patch option -> (annulus bounds, band altitudes, azimuth start, patches per band)
PATCH_LAYOUT = {
    1: ([0, 12, 24, 36, 48, 60, 72, 84, 90], [6, 18, 30, 42, 54, 66, 78, 90],
        [0, 4, 2, 5, 8, 0, 10, 0], [30, 30, 24, 24, 18, 12, 6, 1]),
    2: ([0, 12, 24, 36, 48, 60, 72, 84, 90], [6, 18, 30, 42, 54, 66, 78, 90],
        [0, 4, 2, 5, 8, 0, 10, 0], [31, 30, 28, 24, 19, 13, 7, 1]),
}


# --------------------------------------------------------------- patches
@functools.lru_cache(maxsize=None)
def sky_patches(patch_option: int = 2):
    """(altitude, azimuth) float32 of every sky patch (shadow.py:352-406)."""
    _, altint, azistart, nband = PATCH_LAYOUT[patch_option]
    width = 360 / torch.tensor(nband)
    alt, azi = [], []
    for j, n in enumerate(nband):
        for k in range(n):
            alt.append(float(altint[j]))
            azi.append((k * width[j] + torch.tensor(azistart[j])).item())
    return np.array(alt, F32), np.array(azi, F32)


@functools.lru_cache(maxsize=None)
def sweep_azimuths(patch_option: int = 2) -> np.ndarray:
    """Azimuth the SVF sweep marches for each patch (shadow.py:530-541).

    Each band contributes int(360 / float32(360 / n)) entries, one short of
    n for most bands; the vector starts as zeros, so later patches take the
    shifted azimuths and the last ones keep 0."""
    _, altint, azistart, nband = PATCH_LAYOUT[patch_option]
    width = torch.tensor([360 / p for p in torch.tensor(nband)])
    out = np.zeros(int(sum(nband)), F32)
    i = 0
    for j in range(len(altint)):
        for k in range(int(360 / width[j])):
            v = k * width[j] + torch.tensor(azistart[j])
            if v > 360.:
                v = v - 360.
            out[i] = F32(v.item())
            i += 1
    return out


def _annulus_weight(k: int, n) -> np.float32:
    """Weight of annulus k over n azimuth bins (shadow.py:324-350)."""
    nn = torch.tensor(90.0)
    steprad = (360.0 / n) * (torch.pi / 180.0)
    annulus = 91.0 - torch.tensor(k)
    w = (1.0 / (2.0 * torch.pi)) * torch.sin(torch.pi / (2.0 * nn)) * \
        torch.sin((torch.pi * (2.0 * annulus - 1.0)) / (2.0 * nn))
    return F32((steprad * w).item())


@functools.lru_cache(maxsize=None)
def ring_weights(patch_option: int = 2):
    """Per band: iso and aniso annulus weights (float32), annuli count."""
    annulino, altint, _, nband = PATCH_LAYOUT[patch_option]
    nb = torch.tensor(nband)
    aniso = torch.ceil(nb / 2.0)
    w_iso = np.zeros((N.MAX_RINGS, N.MAX_ANNULI), F32)
    w_an = np.zeros((N.MAX_RINGS, N.MAX_ANNULI), F32)
    count = np.zeros(N.MAX_RINGS, np.int32)
    for i in range(len(altint)):
        ks = range(annulino[i] + 1, annulino[i + 1] + 1)
        count[i] = len(ks)
        for j, k in enumerate(ks):
            w_iso[i, j] = _annulus_weight(k, nb[i])
            w_an[i, j] = _annulus_weight(k, aniso[i])
    return w_iso, w_an, count


# ------------------------------------------------------------ step tables
def _march_steps(branch_y, ssin, scos, tan_a, ds, tanalt, idx):
    """Per-step (dx, dy, dz) for the index vector (float32 arithmetic)."""
    fi = idx.astype(F32)
    m_scos = F32(-1.) * scos
    if branch_y:
        dy = ssin * fi
        dx = m_scos * np.abs(np.rint(fi / tan_a))
    else:
        dy = ssin * np.abs(np.rint(fi * tan_a))
        dx = m_scos * fi
    dz = (ds * fi) * tanalt
    return dx.astype(F32), dy.astype(F32), dz.astype(F32)


def _executed(dx, dy, dz, amax, rows, cols):
    """Number of executed steps: step k runs while the previous step still
    satisfied ``amax >= dz and |dx| < rows and |dy| < cols`` (the first step
    always sees the zero initial state)."""
    ok = (F32(amax) >= dz) & (np.abs(dx) < rows) & (np.abs(dy) < cols)
    if not (F32(amax) >= F32(0.)):
        return 0
    bad = np.flatnonzero(~ok)
    return int(bad[0]) + 1 if bad.size else len(dz)


def step_skip_flags(dx, dy, dz) -> np.ndarray:
    """SW100_STEP_SKIP8 flags of one march's executed steps.  Step k >= 1 is
    flagged when each of the steps k+1 .. k+7 that exist moves at most one
    cell per axis from the step before, and dz does not decrease over the
    steps k-1 .. k+7 (a NaN counts as a decrease).  The kernels' 8-step
    shortcut -- one look-up in a block maximum of the sources over the 3 x 3
    blocks of 8 x 8 cells around step k's cell -- is exact under these two
    facts only; a march whose tables break them is marched step by step."""
    n = len(dz)
    flags = np.zeros(n, np.int32)
    if n < 2:
        return flags
    dx, dy = np.asarray(dx, np.int64), np.asarray(dy, np.int64)
    dz = np.asarray(dz, F32)
    bad_mv = np.zeros(n + 8, np.int64)
    bad_dz = np.zeros(n + 8, np.int64)
    bad_mv[1:n] = (np.abs(np.diff(dx)) > 1) | (np.abs(np.diff(dy)) > 1)
    bad_dz[1:n] = ~(dz[1:] >= dz[:-1])
    cm = np.concatenate([[0], np.cumsum(bad_mv)])  # cm[b] = bad_mv[:b].sum()
    cz = np.concatenate([[0], np.cumsum(bad_dz)])
    k = np.arange(1, n)
    ok = (cm[k + 8] - cm[k + 1] == 0) & (cz[k + 8] - cz[k] == 0)
    flags[1:] = np.where(ok, N.STEP_SKIP8, 0)
    return flags


def _trig(az, alt):
    sin_a, cos_a, tan_a = torch.sin(az), torch.cos(az), torch.tan(az)
    return (F32(torch.sign(sin_a).item()), F32(torch.sign(cos_a).item()), F32(tan_a.item()),
            F32(torch.abs(1. / sin_a).item()), F32(torch.abs(1. / cos_a).item()))


@functools.lru_cache(maxsize=1024)
def _svf_patch_trig(azimuth_deg: float, altitude_deg: int):
    """Site-independent part of a patch march: float32 trigonometry and the
    step-direction branch (shadow.py:196-226)."""
    degrees = torch.pi / 180.
    az = torch.tensor(1e-12) if float(azimuth_deg) == 0.0 else torch.tensor(F32(azimuth_deg))
    alt = torch.tensor(int(altitude_deg))
    az = az * degrees
    alt = alt * degrees
    ssin, scos, tan_a, dssin, dscos = _trig(az, alt)
    pb4 = torch.pi / 4.
    branch_y = bool((pb4 <= az) & (az < 3. * pb4)) or bool((5. * pb4 <= az) & (az < 7. * pb4))
    return branch_y, ssin, scos, tan_a, (dssin if branch_y else dscos), F32(torch.tan(alt).item())


def svf_patch_table(azimuth_deg, altitude_deg, scale, amax, rows, cols):
    """Executed steps of one SVF patch march (shadow.py:196-247)."""
    branch_y, ssin, scos, tan_a, ds, tan_alt = _svf_patch_trig(float(azimuth_deg), int(altitude_deg))
    tanalt = F32(tan_alt / F32(scale))  # float32 tensor / python float
    idx = np.arange(1, max(rows, cols) + 3)
    dx, dy, dz = _march_steps(branch_y, ssin, scos, tan_a, ds, tanalt, idx)
    n = _executed(dx, dy, dz, amax, rows, cols)
    return dx[:n].astype(np.int32), dy[:n].astype(np.int32), dz[:n]


def sun_table(azimuth, altitude, scale, amax, rows, cols):
    """Executed steps of the sun march (solweig.py:1092-1149); returns the
    steps and the float32 azimuth in radians used by the wall tail."""
    degrees = torch.tensor(np.pi / 180.0)
    az = torch.tensor(azimuth) * degrees
    alt = torch.tensor(altitude) * degrees
    ssin, scos, tan_a, dssin, dscos = _trig(az, alt)
    tanalt = F32((torch.tan(alt) / scale).item())
    pb4 = torch.tensor(np.pi / 4.0)
    branch_y = bool((pb4 <= az) & (az < 3 * pb4)) or bool((5 * pb4 <= az) & (az < 7 * pb4))
    ds = dssin if branch_y else dscos
    idx = np.arange(0, max(rows, cols) + 3)
    dx, dy, dz = _march_steps(branch_y, ssin, scos, tan_a, ds, tanalt, idx)
    n = _executed(dx, dy, dz, amax, rows, cols)
    return dx[:n].astype(np.int32), dy[:n].astype(np.int32), dz[:n], F32(az.item())


def sun_tables(azimuths, altitudes, scale, amax, rows, cols):
    """sun_table and facesh_thresholds for every daytime step at once: the
    float32 trigonometry as vectors (each element the same operations as
    the one-step form), the step tables per step.  Returns a list of
    (dx, dy, dz, az_f32, (mode, lo, hi))."""
    if not azimuths:
        return []
    degrees = torch.tensor(np.pi / 180.0)
    az = torch.tensor(list(azimuths)) * degrees
    alt = torch.tensor(list(altitudes)) * degrees
    sin_a, cos_a, tan_a = torch.sin(az), torch.cos(az), torch.tan(az)
    ssin, scos = torch.sign(sin_a).tolist(), torch.sign(cos_a).tolist()
    dssin, dscos = torch.abs(1. / sin_a).tolist(), torch.abs(1. / cos_a).tolist()
    tanalt = (torch.tan(alt) / scale).tolist()
    pb4 = torch.tensor(np.pi / 4.0)
    by = (((pb4 <= az) & (az < 3 * pb4)) | ((5 * pb4 <= az) & (az < 7 * pb4))).tolist()
    # wall-face bounds (facesh_thresholds) on the float32 azimuths
    lo = az - torch.pi / 2
    hi = az + torch.pi / 2
    mode0 = ((lo >= 0) & (hi < 2 * torch.pi)).tolist()
    up = ((lo < 0) & (hi <= 2 * torch.pi)).tolist()
    down = ((lo > 0) & (hi >= 2 * torch.pi)).tolist()
    lo_up, hi_down = (lo + 2 * torch.pi).tolist(), (hi - 2 * torch.pi).tolist()
    lo_l, hi_l, az_l, tan_l = lo.tolist(), hi.tolist(), az.tolist(), tan_a.tolist()
    consts = np.zeros(len(az_l), N.MARCH_CONST_DTYPE)
    consts["branch_y"] = by
    consts["ssin"], consts["scos"], consts["tan_a"] = ssin, scos, tan_l
    consts["ds"] = [dssin[k] if by[k] else dscos[k] for k in range(len(az_l))]
    consts["tanalt"] = tanalt
    steps, counts = N.march_tables(consts, 0, amax, rows, cols)
    offs = np.concatenate([[0], np.cumsum(counts)])
    out = []
    for k in range(len(az_l)):
        t = steps[offs[k]:offs[k + 1]]
        if mode0[k]:
            face = (0, F32(lo_l[k]), F32(hi_l[k]))
        elif up[k]:
            face = (1, F32(lo_up[k]), F32(hi_l[k]))
        elif down[k]:
            face = (1, F32(lo_l[k]), F32(hi_down[k]))
        else:
            raise ValueError(f"sun azimuth {az_l[k]} outside the wall-face branches")
        out.append((t["dx"].copy(), t["dy"].copy(), t["dz"].copy(), F32(az_l[k]), face))
    return out


def facesh_thresholds(az_rad_f32):
    """Branch and float32 bounds of the wall-face test (solweig.py:1187-1196,
    :239-248): mode 0 -> facesh = [aspect < lo or aspect >= hi] - wallbol + 1,
    mode 1 -> facesh = 1 - [aspect > lo or aspect <= hi]."""
    azt = torch.tensor(F32(az_rad_f32))
    lo = azt - torch.pi / 2
    hi = azt + torch.pi / 2
    if lo >= 0 and hi < 2 * torch.pi:
        return 0, F32(lo.item()), F32(hi.item())
    if lo < 0 and hi <= 2 * torch.pi:
        lo = lo + 2 * torch.pi
    elif lo > 0 and hi >= 2 * torch.pi:
        hi = hi - 2 * torch.pi
    else:
        raise ValueError(f"sun azimuth {az_rad_f32} outside the wall-face branches")
    return 1, F32(lo.item()), F32(hi.item())


@functools.lru_cache(maxsize=None)
def gvf_table(second: int) -> np.ndarray:
    """Walk offsets and face bounds of the 18 ground-view-factor azimuths."""
    if second > N.MAX_GVF_STEPS:
        raise ValueError(f"ground view factor walk of {second} steps exceeds {N.MAX_GVF_STEPS}")
    tab = np.zeros(N.N_GVF_AZ, N.GVF_AZ_DTYPE)
    azs = np.arange(5, 359, 20, dtype=np.float32)
    for j, a in enumerate(azs):
        az = torch.tensor(a) * (torch.pi / 180)
        ssin, scos, tan_a, _, _ = _trig(az, az)
        pb4 = torch.pi / 4
        branch_y = bool((pb4 <= az) & (az < 3 * pb4)) or bool((5 * pb4 <= az) & (az < 7 * pb4))
        dx, dy, _ = _march_steps(branch_y, ssin, scos, tan_a, F32(0), F32(0), np.arange(second))
        tab["dx"][j, :second] = dx.astype(np.int8)
        tab["dy"][j, :second] = dy.astype(np.int8)
        mode, lo, hi = facesh_thresholds(F32(az.item()))
        tab["facesh_mode"][j], tab["facesh_lo"][j], tab["facesh_hi"][j] = mode, lo, hi
        flags = 0
        if 0 <= a < 180:
            flags |= 1
        if 90 <= a < 270:
            flags |= 2
        if 180 <= a < 360:
            flags |= 4
        if 270 <= a or a < 90:
            flags |= 8
        tab["dir_flags"][j] = flags
    return tab


def svf_plan(rows, cols, scale, amax, bush_any, patch_option=2, trans_veg=0.03, all_finite=False):
    """SVF plan record + concatenated step table + single-step patch mask."""
    annulino, altint, _, nband = PATCH_LAYOUT[patch_option]
    w_iso, w_an, count = ring_weights(patch_option)
    plan = np.zeros(1, N.SVF_PLAN_DTYPE)
    P = int(sum(nband))
    plan["n_patches"] = P
    plan["n_rings"] = len(altint)
    plan["bush_any"] = int(bool(bush_any))
    plan["all_finite"] = int(bool(all_finite))
    plan["ring_annuli"][0, :] = count
    plan["w_iso"][0] = w_iso
    plan["w_aniso"][0] = w_an
    plan["tail"] = F32(3.0459e-004)
    plan["trans"] = F32(0.03)
    plan["trans_veg"] = F32(trans_veg)
    ring, consts, tan_alt, dir_flags = _svf_layout(patch_option)
    steps, counts = _svf_steps_all(consts, tan_alt, scale, amax, rows, cols)
    single = np.zeros(N.CUBE_WORDS, np.uint32)
    offsets = np.concatenate([[0], np.cumsum(counts)[:-1]]) if P else np.zeros(0, np.int64)
    plan["step_offset"][0, :P] = offsets
    plan["step_count"][0, :P] = counts
    plan["ring"][0, :P] = ring
    plan["dir_flags"][0, :P] = dir_flags
    for q in np.flatnonzero(np.asarray(counts) <= 1):
        single[q >> 5] |= np.uint32(1 << (int(q) & 31))
    return plan, steps, single


@functools.lru_cache(maxsize=None)
def _svf_layout(patch_option):
    """The site-independent part of the SVF plan of a patch layout: each
    patch's ring, march constants (float32 trigonometry and step-direction
    branch, shadow.py:196-226) without the scale-dependent tan(altitude),
    tan(altitude) itself, and its direction-sum flags (E, S, W, N)."""
    _, altint, _, nband = PATCH_LAYOUT[patch_option]
    P = int(sum(nband))
    azs = sweep_azimuths(patch_option)[:P]
    ring = np.repeat(np.arange(len(altint)), nband)[:P]
    trig = [_svf_patch_trig(float(a), int(h)) for a, h in zip(azs, np.asarray(altint)[ring])]
    consts = np.zeros(len(trig), N.MARCH_CONST_DTYPE)
    consts["branch_y"] = [t[0] for t in trig]
    consts["ssin"] = [t[1] for t in trig]
    consts["scos"] = [t[2] for t in trig]
    consts["tan_a"] = [t[3] for t in trig]
    consts["ds"] = [t[4] for t in trig]
    tan_alt = np.array([t[5] for t in trig], np.float32)
    dir_flags = np.array([((1 if 0 <= a < 180 else 0) | (2 if 90 <= a < 270 else 0) | (4 if 180 <= a < 360 else 0) |
                           (8 if (a >= 270 or a < 90) else 0)) for a in map(float, azs)], np.int32)
    for a in (ring, consts, tan_alt, dir_flags):
        a.setflags(write=False)
    return ring, consts, tan_alt, dir_flags


def _svf_steps_all(consts, tan_alt, scale, amax, rows, cols):
    """Executed steps of every patch march at once, concatenated in patch
    order with their SW100_STEP_SKIP8 flags (sw100_march_tables: the same
    float32 values as svf_patch_table applied patch by patch); returns
    (steps, counts)."""
    c = consts.copy()
    c["tanalt"] = tan_alt / F32(scale)      # float32 / float32, per element as F32(t / F32(scale))
    return N.march_tables(c, 1, amax, rows, cols)


# ------------------------------------------- windowed SVF recompute
def svf_corridor(plan: np.ndarray, steps: np.ndarray, height_bound: float):
    """Corridor descriptors of the windowed recompute, one int32 per patch.

    A patch whose step k shifts by s * (k + 1) along one axis (its major
    axis) and whose other shift changes by at most one cell per step, in one
    direction, gets ``axis | (4 if s < 0)``.  A patch whose every step drops
    the source by more than twice ``height_bound`` (the largest |height| of
    the march rasters before and after the edit) gets ``CORRIDOR_LOCAL``:
    every in-grid source then shades the pixel whatever its height (the
    zenith patch, whose float32 tan(90 deg) is a large negative number), so
    only pixels inside the edit re-march it.  Any other table gets
    ``CORRIDOR_ALWAYS`` (re-marched by every window pixel).  The device test
    (csrc/svf_sweep.cu svf_in_corridor) relies on exactly these properties."""
    n_p = int(plan["n_patches"][0])
    desc = np.full(n_p, N.CORRIDOR_ALWAYS, np.int32)
    blind = -(2.0 * float(height_bound) + 16.0)
    for q in range(n_p):
        off, n = int(plan["step_offset"][0, q]), int(plan["step_count"][0, q])
        dx = steps["dx"][off:off + n].astype(np.int64)
        dy = steps["dy"][off:off + n].astype(np.int64)
        dz = steps["dz"][off:off + n].astype(np.float64)
        if n == 0 or np.all(dz < blind):
            desc[q] = N.CORRIDOR_LOCAL
            continue
        k1 = np.arange(1, n + 1)
        for axis, major, minor in ((0, dx, dy), (1, dy, dx)):
            s = 1 if np.array_equal(major, k1) else (-1 if np.array_equal(major, -k1) else 0)
            if s == 0:
                continue
            d = np.diff(minor)
            if np.all(np.abs(d) <= 1) and (np.all(d >= 0) or np.all(d <= 0)):
                desc[q] = axis | (4 if s < 0 else 0)
                break
    return desc


def in_corridor(desc: int, dx: np.ndarray, dy: np.ndarray, t, rect) -> bool:
    """Host restatement of the device corridor test (svf_in_corridor)."""
    tr, tc = t
    r0, r1, c0, c1 = rect
    if r0 <= tr <= r1 and c0 <= tc <= c1:
        return True
    n = len(dx)
    axis = desc & 3
    if n == 0 or axis == N.CORRIDOR_LOCAL:
        return False
    if axis == N.CORRIDOR_ALWAYS:
        return True
    neg = bool(desc & 4)
    tM, lo, hi = (tr, r0, r1) if axis == 0 else (tc, c0, c1)
    tm, mlo, mhi = (tc, c0, c1) if axis == 0 else (tr, r0, r1)
    ka = max(tM - hi if neg else lo - tM, 1)
    kb = min(tM - lo if neg else hi - tM, n)
    if ka > kb:
        return False
    minor = dy if axis == 0 else dx
    ma, mb = int(minor[ka - 1]), int(minor[kb - 1])
    return tm + max(ma, mb) >= mlo and tm + min(ma, mb) <= mhi


def edit_window(rect, plan: np.ndarray, steps: np.ndarray, desc: np.ndarray, rows: int, cols: int):
    """Pixels whose marches can read the edited rectangle: the rectangle
    and, per patch that is not local, the rectangle shifted back by every
    executed step (a box per patch), clipped to the grid; inclusive bounds."""
    r0, r1, c0, c1 = rect
    w = [r0, r1, c0, c1]
    for q in range(len(desc)):
        if (desc[q] & 3) == N.CORRIDOR_LOCAL:
            continue
        off, n = int(plan["step_offset"][0, q]), int(plan["step_count"][0, q])
        dx = steps["dx"][off:off + n]
        dy = steps["dy"][off:off + n]
        w[0] = min(w[0], r0 - int(dx.max()))
        w[1] = max(w[1], r1 - int(dx.min()))
        w[2] = min(w[2], c0 - int(dy.max()))
        w[3] = max(w[3], c1 - int(dy.min()))
    return (max(0, w[0]), min(rows - 1, w[1]), max(0, w[2]), min(cols - 1, w[3]))


def patch_shift_bounds(plan: np.ndarray, steps: np.ndarray, desc: np.ndarray) -> np.ndarray:
    """(min dx, max dx, min dy, max dy) over the executed steps of every
    patch that is not local (rows of zeros for the others)."""
    out = np.zeros((len(desc), 4), np.int64)
    for q in range(len(desc)):
        if (desc[q] & 3) == N.CORRIDOR_LOCAL:
            continue
        off, n = int(plan["step_offset"][0, q]), int(plan["step_count"][0, q])
        dx, dy = steps["dx"][off:off + n], steps["dy"][off:off + n]
        out[q] = (dx.min(), dx.max(), dy.min(), dy.max())
    return out


def window_from_bounds(rect, bounds: np.ndarray, rows: int, cols: int):
    """:func:`edit_window` from the per-patch shift bounds."""
    r0, r1, c0, c1 = rect
    return (max(0, r0 - int(bounds[:, 1].max(initial=0))), min(rows - 1, r1 - int(bounds[:, 0].min(initial=0))),
            max(0, c0 - int(bounds[:, 3].max(initial=0))), min(cols - 1, c1 - int(bounds[:, 2].min(initial=0))))


# ----------------------------------------------------- predicate bounds
def _f32_to_key(x):
    b = np.asarray(x, F32).view(np.int32).astype(np.int64)
    return np.where(b >= 0, b, -(b & 0x7FFFFFFF))


def _key_to_f32(k):
    k = np.asarray(k, np.int64)
    b = np.where(k >= 0, k, (-k) | 0x80000000).astype(np.uint32)
    return b.view(F32)


@functools.lru_cache(maxsize=None)
def atan_degree_bounds(palt: float):
    """Bounds on tan_delta for the shaded_or_sunlit predicate
    (solweig.py:524-562): with g(x) = float32(atan(x) * (180 / pi)) evaluated
    by torch's CPU kernel,  sunlit <=> x < lo  and  shaded <=> x > hi, where
    lo = min{x : g(x) >= palt} and hi = max{x : g(x) <= palt}.  g is monotone;
    both bounds are found by bisection over the ordered float32 values."""
    palt = F32(palt)
    rad2deg = 180.0 / torch.pi

    def g(keys):
        x = torch.from_numpy(_key_to_f32(keys).copy())
        return (torch.atan(x) * rad2deg).numpy()

    inf_key = int(_f32_to_key(F32(np.inf)))

    def search(pred):  # smallest key with pred(g) true (monotone false -> true)
        lo, hi = -inf_key, inf_key
        if not pred(g(np.array([hi])))[0]:
            return None
        while hi - lo > 1:
            mid = (lo + hi) // 2
            if pred(g(np.array([mid])))[0]:
                hi = mid
            else:
                lo = mid
        return hi

    k_lo = search(lambda v: v >= palt)
    k_gt = search(lambda v: v > palt)
    lo = F32(np.inf) if k_lo is None else _key_to_f32(np.array([k_lo]))[0]
    hi = F32(np.inf) if k_gt is None else _key_to_f32(np.array([k_gt - 1]))[0]
    return F32(lo), F32(hi)
