"""Build the sm_100a shared library ``libsolweig_b200.so`` in-tree with nvcc.

    python -m solweig_project_b200.build [--force] [--verbose]

Every kernel is compiled with ``--fmad=false`` (no contracted multiply-adds:
the reference's float32 operation sequence is reproduced one rounding at a
time) and IEEE division / square root.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(REPO, "include")
LIB_NAME = "libsolweig_b200.so"
LIB_PATH = os.path.join(PKG, LIB_NAME)
SOURCES = ("api.cu", "prepare.cu", "svf_sweep.cu", "sun_march.cu", "time_loop.cu", "utci.cu", "nn.cu",
           "patch_sums.cu")
ARCH = "-gencode=arch=compute_100a,code=sm_100a"
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "--prec-div=true", "--prec-sqrt=true",
         "--ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", "-Xptxas", "-v"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def write_utci_include() -> str:
    """Generate csrc/utci_series.inc from data/utci_terms.json: one
    SW_UTCI_TERM(j, pt, pv, pd, pp, c) line per regression term, in the
    reference's summation order, with c rounded to float32 (written as an
    exact hexadecimal literal)."""
    import numpy as np
    with open(os.path.join(PKG, "data", "utci_terms.json")) as fh:
        terms = json.load(fh)["terms"]
    lines = [f"SW_UTCI_TERM({j}, {a}, {b}, {d}, {e}, {float(np.float32(float(c))).hex()}f)"
             for j, (c, a, b, d, e) in enumerate(terms)]
    text = "// generated from solweig_project_b200/data/utci_terms.json\n" + "\n".join(lines) + "\n"
    path = os.path.join(CSRC, "utci_series.inc")
    old = open(path).read() if os.path.exists(path) else None
    if old != text:
        with open(path, "w") as fh:
            fh.write(text)
    return path


def _digest(paths) -> str:
    h = hashlib.sha256()
    for p in paths:
        with open(p, "rb") as fh:
            h.update(fh.read())
    h.update(" ".join(FLAGS + [ARCH]).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> str:
    inc = write_utci_include()
    deps = [os.path.join(CSRC, s) for s in SOURCES]
    deps += [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cuh", ".inc"))]
    deps += [os.path.join(INCLUDE, "solweig_b200.h"), inc]
    digest = _digest(deps)
    stamp = LIB_PATH + ".sha256"
    if not force and os.path.exists(LIB_PATH) and os.path.exists(stamp):
        if open(stamp).read().strip() == digest:
            return LIB_PATH
    cmd = [nvcc(), ARCH, *FLAGS, "-I", INCLUDE, "-I", CSRC, "-o", LIB_PATH + ".tmp",
           *[os.path.join(CSRC, s) for s in SOURCES]]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode})")
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    with open(stamp, "w") as fh:
        fh.write(digest + "\n")
    with open(os.path.join(PKG, "ptxas_info.txt"), "w") as fh:
        fh.write(res.stderr)
    return LIB_PATH


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose))


if __name__ == "__main__":
    main()
