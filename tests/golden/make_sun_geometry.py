"""Sun geometry of the benchmark workloads, computed with the reference's own
``Solweig_2015a_metdata_noload`` (solweig_gpu/sun_position.py:905-1010).

    python tests/golden/make_sun_geometry.py --ref <reference checkout>

(``--ref`` may be replaced by the environment variable ``SOLWEIG_REFERENCE``.)

Writes tests/golden/sun_geometry.npz with, per site, the float64 (1, 24)
arrays altitude / azimuth / zen / jday / dectime / altmax that
run_utci_window takes, for:

* ``single``: the single-site workloads (lat 30.3, lon -97.7, altitude 3 m,
  UTC-5, seed 1234 forcing);
* ``multi``: the 64-site batched workload (seeded latitudes U(0, 60), each
  site with the forcing of its own seed, see ``multi_site_specs``).
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from make_golden import install_stubs, reference_path  # noqa: E402
from solweig_project_b200 import synthetic  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference checkout (or $SOLWEIG_REFERENCE)")
    args = ap.parse_args()
    install_stubs(reference_path(args.ref))
    import solweig_gpu.sun_position as rsun
    out = {}

    def geometry(prefix, met, loc):
        _, alt, azi, zen, jday, _, dectime, altmax = rsun.Solweig_2015a_metdata_noload(met, loc, synthetic.DEFAULT_UTC)
        for k, v in (("altitude", alt), ("azimuth", azi), ("zen", zen), ("jday", jday), ("dectime", dectime),
                     ("altmax", altmax)):
            out[f"{prefix}_{k}"] = np.asarray(v, np.float64)

    geometry("single", synthetic.make_met(1234), dict(synthetic.DEFAULT_LOCATION))
    specs = synthetic.multi_site_specs()
    for i, s in enumerate(specs):
        loc = {"latitude": s["latitude"], "longitude": s["longitude"], "altitude": 3.0}
        geometry(f"multi{i}", synthetic.make_met(s["seed"]), loc)
    path = os.path.join(HERE, "sun_geometry.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e3:.1f} kB)")


if __name__ == "__main__":
    main()
