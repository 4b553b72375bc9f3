"""Oracle: SVF patch sweep (reference ``solweig_gpu/shadow.py``).

* :func:`create_patches` -- ``shadow.py:352-406`` (sky vault patch layout)
* :func:`annulus_weight` -- ``shadow.py:324-350``
* :func:`shadow_step_table` -- the scalar part of ``shadow.py:166-247``
  (per-step shifts and height drops of one patch march)
* :func:`shadow_patch` -- ``shadow.py:166-322`` (one patch march over planes)
* :func:`svf_calculator` -- ``shadow.py:409-625`` (153-patch sweep + sums),
  split into :func:`patch_tasks`, the marches and :class:`SvfAccumulator`
"""
from __future__ import annotations

import numpy as np
import torch

F32 = np.float32

_PATCH_LAYOUT = {
    # option: (annulino, altitude bands, azimuth start, patches per band)
    1: ([0, 12, 24, 36, 48, 60, 72, 84, 90], [6, 18, 30, 42, 54, 66, 78, 90],
        [0, 4, 2, 5, 8, 0, 10, 0], [30, 30, 24, 24, 18, 12, 6, 1]),
    2: ([0, 12, 24, 36, 48, 60, 72, 84, 90], [6, 18, 30, 42, 54, 66, 78, 90],
        [0, 4, 2, 5, 8, 0, 10, 0], [31, 30, 28, 24, 19, 13, 7, 1]),
    3: ([0, 12, 24, 36, 48, 60, 72, 84, 90], [6, 18, 30, 42, 54, 66, 78, 90],
        [0, 4, 2, 5, 8, 0, 10, 0], [62, 60, 56, 48, 38, 26, 14, 1]),
}


def create_patches(patch_option: int = 2):
    """Patch altitudes/azimuths (float32) and band layout (shadow.py:352-406)."""
    annulino, altint, azistart, nband = _PATCH_LAYOUT[patch_option]
    nband_t = torch.tensor(nband)
    aziint = 360 / nband_t  # float32 band widths
    alt, azi = [], []
    for j in range(len(altint)):
        for k in range(nband[j]):
            alt.append(torch.tensor([altint[j]], dtype=torch.float32))
            azi.append((k * aziint[j] + torch.tensor(azistart[j])).reshape(1).float())
    return (torch.cat(alt).numpy(), torch.cat(azi).numpy(), np.array(annulino), np.array(altint),
            np.array(nband), aziint.numpy(), np.array(azistart))


def annulus_weight(k: int, n) -> np.float32:
    """Solid-angle weight of annulus ``k`` split over ``n`` azimuth bins
    (shadow.py:324-350); ``n`` is an int64 (iso) or float32 (aniso) 0-dim
    tensor as in the reference."""
    nn = torch.tensor(90.0)
    altitude = torch.tensor(k)
    steprad = (360.0 / n) * (torch.pi / 180.0)
    annulus = 91.0 - altitude
    w = (1.0 / (2.0 * torch.pi)) * torch.sin(torch.pi / (2.0 * nn)) * \
        torch.sin((torch.pi * (2.0 * annulus - 1.0)) / (2.0 * nn))
    return F32((steprad * w).item())


def patch_azimuths(patch_option: int = 2) -> np.ndarray:
    """``iazimuth`` of svf_calculator (shadow.py:530-541), float32.

    The per-band count is ``int(360 / float32(360 / n))``, which truncates to
    ``n - 1`` for several bands; the vector is pre-filled with zeros, so the
    later patches take shifted azimuths and the last few keep azimuth 0."""
    annulino, altint, azistart, nband = _PATCH_LAYOUT[patch_option]
    aziint = torch.tensor([360 / p for p in torch.tensor(nband)])
    out = np.zeros(int(sum(nband)), np.float32)
    index = 0
    for j in range(len(altint)):
        for k in range(int(360 / aziint[j])):
            v = k * aziint[j] + torch.tensor(azistart[j])
            if v > 360.:
                v = v - 360.
            out[index] = F32(v.item())
            index += 1
    return out


def shadow_step_table(azimuth_deg, altitude_deg, scale, amaxvalue, rows, cols):
    """Executed (dx, dy, dz) sequence of one ``shadow()`` march.

    ``azimuth_deg`` is the float32 patch azimuth, ``altitude_deg`` the integer
    band altitude.  Trigonometry runs on 0-dim float32 torch tensors exactly as
    in shadow.py:196-226; the per-step arithmetic is IEEE float32
    (shadow.py:230-239).  Returns int arrays dx, dy and float32 dz.
    """
    degrees = torch.pi / 180.
    if float(azimuth_deg) == 0.0:
        az = torch.tensor(1e-12)
    else:
        az = torch.tensor(F32(azimuth_deg))
    alt = torch.tensor(int(altitude_deg)) if float(altitude_deg).is_integer() \
        else torch.tensor(F32(altitude_deg))
    az = az * degrees
    alt = alt * degrees
    sin_a, cos_a, tan_a = torch.sin(az), torch.cos(az), torch.tan(az)
    ssin, scos = torch.sign(sin_a), torch.sign(cos_a)
    dssin = torch.abs(1. / sin_a)
    dscos = torch.abs(1. / cos_a)
    tanalt = torch.tan(alt) / scale
    pb4 = torch.pi / 4.
    branch_y = bool((pb4 <= az) & (az < 3. * pb4)) or bool((5. * pb4 <= az) & (az < 7. * pb4))
    tan_a, ssin, scos = F32(tan_a.item()), F32(ssin.item()), F32(scos.item())
    ds = F32(dssin.item()) if branch_y else F32(dscos.item())
    tanalt = F32(tanalt.item())
    amax = F32(amaxvalue)
    m_scos = F32(-1.) * scos
    dxs, dys, dzs = [], [], []
    dx = dy = dz = F32(0.)
    index = 1
    while amax >= dz and abs(dx) < rows and abs(dy) < cols:
        fi = F32(index)
        if branch_y:
            dy = ssin * fi
            dx = m_scos * np.abs(np.rint(fi / tan_a))
        else:
            dy = ssin * np.abs(np.rint(fi * tan_a))
            dx = m_scos * fi
        dz = (ds * fi) * tanalt
        dxs.append(int(dx))
        dys.append(int(dy))
        dzs.append(dz)
        index += 1
    return np.array(dxs, np.int64), np.array(dys, np.int64), np.array(dzs, np.float32)


def _shift(plane, dx, dy, fill=0.0):
    """``out[r, c] = plane[r + dx, c + dy]`` where in bounds, else ``fill``."""
    rows, cols = plane.shape
    out = np.full_like(plane, fill)
    r0, r1 = max(0, -dx), min(rows, rows - dx)
    c0, c1 = max(0, -dy), min(cols, cols - dy)
    if r0 < r1 and c0 < c1:
        out[r0:r1, c0:c1] = plane[r0 + dx:r1 + dx, c0 + dy:c1 + dy]
    return out


def torch_max(x, y):
    """``torch.max(x, y)``: NaN propagates; on ties the second operand wins."""
    return np.where((x > y) | np.isnan(x), x, y)


def shadow_patch(amaxvalue, a, vegdem, vegdem2, bush, azimuth_deg, altitude_deg, scale):
    """One SVF patch march (shadow.py:166-322) -> (sh, vegsh, vbshvegsh)."""
    rows, cols = a.shape
    dxs, dys, dzs = shadow_step_table(azimuth_deg, altitude_deg, scale, amaxvalue, rows, cols)
    f = a.copy()
    g = np.zeros_like(a)
    sh = np.zeros_like(a)
    vbshvegsh = np.zeros_like(a)
    bushplant = (bush > 1.).astype(F32)
    vegsh = np.zeros_like(a) + bushplant
    bush_any = bool(bush.max() > 0.) if bush.size else False
    for step, (dx, dy, dz) in enumerate(zip(dxs, dys, dzs)):
        inb = _shift(np.ones_like(a), dx, dy)
        tempvegdem = np.where(inb > 0, _shift(vegdem, dx, dy) - dz, F32(0.)).astype(F32)
        tempvegdem2 = np.where(inb > 0, _shift(vegdem2, dx, dy) - dz, F32(0.)).astype(F32)
        temp = np.where(inb > 0, _shift(a, dx, dy) - dz, F32(0.)).astype(F32)
        f = torch_max(f, temp)
        sh = np.where(f > a, F32(1.), np.where(f <= a, F32(0.), sh)).astype(F32)
        fabovea = tempvegdem > a
        gabovea = tempvegdem2 > a
        vegsh2 = fabovea.astype(F32) - gabovea.astype(F32)
        vegsh = torch_max(vegsh, vegsh2)
        vegsh[(vegsh * sh) > 0.] = 0.
        vbshvegsh = vegsh + vbshvegsh
        if step == 0:
            firstvegdem = tempvegdem - temp
            firstvegdem[firstvegdem <= 0.] = 1000.
            vegsh[firstvegdem < dz] = 1.
            vegsh = vegsh * (vegdem2 > a).astype(F32)
            vbshvegsh[...] = 0.
        if bush_any and float(np.max(fabovea * bush)) > 0.:
            tempbush = np.where(inb > 0, _shift(bush, dx, dy) - dz, F32(0.)).astype(F32)
            g = torch_max(g, tempbush)
            g = g * bushplant
    sh = F32(1.) - sh
    vbshvegsh[vbshvegsh > 0.] = 1.
    vbshvegsh = vbshvegsh - vegsh
    if bush_any:
        g = g - bush
        g[g > 0.] = 1.
        g[g < 0.] = 0.
        vegsh = vegsh - bushplant + g
        vegsh[vegsh < 0.] = 0.
    vegsh[vegsh > 0.] = 1.
    vegsh = F32(1.) - vegsh
    vbshvegsh = F32(1.) - vbshvegsh
    return sh.astype(F32), vegsh.astype(F32), vbshvegsh.astype(F32), len(dzs)


SVF_ORDER = ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg",
             "svfS", "svfSaveg", "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg",
             "vegshmat", "vbshvegshmat", "shmat", "svftotal")


def patch_tasks(patch_option=2):
    """The patches of the sweep in the reference's order (shadow.py:447-620):
    (index, band, azimuth, altitude) per patch, the values passed to the
    march exactly as svf_calculator passes them."""
    annulino, altint, _, nband = _PATCH_LAYOUT[patch_option]
    iaz = patch_azimuths(patch_option)
    out, index = [], 0
    for i in range(len(altint)):
        for _ in range(nband[i]):
            out.append((index, i, iaz[index], altint[i]))
            index += 1
    return out


class SvfAccumulator:
    """The sums of svf_calculator (shadow.py:447-625) fed one patch at a time,
    in patch order; the marches themselves (shadow_patch) are independent and
    may run anywhere, in any order."""

    def __init__(self, patch_option, rows, cols, vegdem2):
        z = lambda: np.zeros((rows, cols), F32)  # noqa: E731
        self.planes = {k: z() for k in ("svf", "svfE", "svfS", "svfW", "svfN", "svfveg", "svfEveg", "svfSveg",
                                        "svfWveg", "svfNveg", "svfaveg", "svfEaveg", "svfSaveg", "svfWaveg",
                                        "svfNaveg")}
        self.annulino, self.altint, _, self.nband = _PATCH_LAYOUT[patch_option]
        P = int(sum(self.nband))
        self.shmat = np.zeros((rows, cols, P), F32)
        self.vegshmat = np.zeros((rows, cols, P), F32)
        self.vbshmat = np.zeros((rows, cols, P), F32)
        nband_t = torch.tensor(self.nband)
        aniso_t = torch.ceil(nband_t / 2.0)
        an = self.annulino
        self.w_iso = [{k: annulus_weight(k, nband_t[i]) for k in range(an[i] + 1, an[i + 1] + 1)}
                      for i in range(len(self.altint))]
        self.w_an = [{k: annulus_weight(k, aniso_t[i]) for k in range(an[i] + 1, an[i + 1] + 1)}
                     for i in range(len(self.altint))]
        self.vegdem2 = vegdem2
        self.next = 0
        self.steps = []

    def add(self, task, sh, vegsh, vbsh, nst):
        index, i, az, _ = task
        if index != self.next:
            raise ValueError(f"patch {index} added out of order (expected {self.next})")
        self.next += 1
        self.steps.append(nst)
        self.shmat[:, :, index] = sh
        self.vegshmat[:, :, index] = vegsh
        self.vbshmat[:, :, index] = vbsh
        P = self.planes
        inE = 0 <= az < 180
        inS = 90 <= az < 270
        inW = 180 <= az < 360
        inN = az >= 270 or az < 90
        for k in range(self.annulino[i] + 1, self.annulino[i + 1] + 1):
            wi, wa = self.w_iso[i][k], self.w_an[i][k]
            P["svf"] = P["svf"] + wi * sh
            wsh = wa * sh
            if inE:
                P["svfE"] = P["svfE"] + wsh
            if inS:
                P["svfS"] = P["svfS"] + wsh
            if inW:
                P["svfW"] = P["svfW"] + wsh
            if inN:
                P["svfN"] = P["svfN"] + wsh
            P["svfveg"] = P["svfveg"] + wi * vegsh
            P["svfaveg"] = P["svfaveg"] + wi * vbsh
            for d, on in (("E", inE), ("S", inS), ("W", inW), ("N", inN)):
                if on:
                    P[f"svf{d}veg"] = P[f"svf{d}veg"] + wa * vegsh
                    P[f"svf{d}aveg"] = P[f"svf{d}aveg"] + wa * vbsh

    def result(self):
        """The reference's 19-tuple once every patch has been added."""
        if self.next != self.shmat.shape[2]:
            raise ValueError(f"{self.next} of {self.shmat.shape[2]} patches added")
        P = dict(self.planes)
        tail = F32(3.0459e-004)
        P["svfS"] = P["svfS"] + tail
        P["svfW"] = P["svfW"] + tail
        for k in ("svf", "svfE", "svfS", "svfW", "svfN"):
            P[k][P[k] > 1.] = 1.
        last = np.zeros_like(P["svf"])
        last[self.vegdem2 == 0.] = tail
        for k in ("svfSveg", "svfWveg", "svfSaveg", "svfWaveg"):
            P[k] = P[k] + last
        for k in ("svfveg", "svfEveg", "svfSveg", "svfWveg", "svfNveg", "svfaveg", "svfEaveg", "svfSaveg",
                  "svfWaveg", "svfNaveg"):
            P[k][P[k] > 1.] = 1.
        trans = F32(0.03)
        svftotal = P["svf"] - (F32(1) - P["svfveg"]) * (F32(1) - trans)
        return tuple(P[k] for k in ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg",
                                    "svfNveg", "svfS", "svfSaveg", "svfSveg", "svfveg", "svfW", "svfWaveg",
                                    "svfWveg")) + (self.vegshmat, self.vbshmat, self.shmat, svftotal)


def svf_calculator(patch_option, amaxvalue, a, vegdem, vegdem2, bush, scale, return_steps=False, march_map=None):
    """153-patch sweep (shadow.py:409-625); returns the reference's 19-tuple
    (15 SVF planes, 3 (rows, cols, P) cubes, SVFtotal).  ``march_map(tasks)``
    (optional) yields (task, (sh, vegsh, vbsh, n_steps)) in task order for
    the scene of this call -- e.g. a process pool set up by march_pool --
    instead of marching the patches here one after another."""
    a = np.asarray(a, F32)
    vegdem = np.asarray(vegdem, F32)
    vegdem2 = np.asarray(vegdem2, F32)
    bush = np.asarray(bush, F32)
    rows, cols = a.shape
    acc = SvfAccumulator(patch_option, rows, cols, vegdem2)
    tasks = patch_tasks(patch_option)
    if march_map is None:
        for t in tasks:
            acc.add(t, *shadow_patch(amaxvalue, a, vegdem, vegdem2, bush, t[2], t[3], scale))
    else:
        for t, res in march_map(tasks):
            acc.add(t, *res)
    out = acc.result()
    if return_steps:
        return out, np.array(acc.steps)
    return out


# ---- patch marches in worker processes (the CPU timing of the sweep on all
# host cores; the sums stay in the parent, in patch order, so the result is
# the serial sweep's bit for bit)
_SCENE = None


def _march_init(scene):
    global _SCENE
    torch.set_num_threads(1)   # one process per core
    _SCENE = scene


def _ready(_):
    import os
    return os.getpid()


def _march_one(task):
    amaxvalue, a, vegdem, vegdem2, bush, scale = _SCENE
    return task, shadow_patch(amaxvalue, a, vegdem, vegdem2, bush, task[2], task[3], scale)


def march_pool(processes, amaxvalue, a, vegdem, vegdem2, bush, scale):
    """A spawn-started process pool holding one scene; ``pool.imap(
    march_one, tasks)`` marches its patches.  Returns (pool, march_one)."""
    import multiprocessing as mp
    scene = (amaxvalue, np.asarray(a, F32), np.asarray(vegdem, F32), np.asarray(vegdem2, F32),
             np.asarray(bush, F32), scale)
    pool = mp.get_context("spawn").Pool(processes, initializer=_march_init, initargs=(scene,))
    pool.map(_ready, range(4 * processes), chunksize=1)   # every worker started and holding the scene
    return pool, _march_one


def scene_from_rasters(dsm, trees, dem):
    """Derived march inputs exactly as compute_utci builds them
    (utci_process.py:1377-1385): vegdsm, vegdsm2, bush, amaxvalue."""
    a = np.asarray(dsm, F32)
    t1 = np.asarray(trees, F32).copy()
    t2 = np.asarray(dem, F32)
    t1[t1 < 0.] = 0.
    vegdem = t1 + t2
    vegdem2 = t1 * F32(0.25) + t2
    bush = np.logical_not(vegdem2 * vegdem).astype(F32) * vegdem
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * F32(0.25) + a
    vegdsm2[vegdsm2 == a] = 0
    amax = F32(max(a.max(), vegdem.max()))
    return vegdsm.astype(F32), vegdsm2.astype(F32), bush.astype(F32), amax
