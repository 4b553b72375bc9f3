"""Writes spa_terms.json: the periodic-term tables of the Solar Position
Algorithm (Reda, I. and Andreas, A., 2004, "Solar position algorithm for
solar radiation applications", Solar Energy 76(5):577-589, NREL/TP-560-34302,
Tables A4.2 and A4.3: the Earth heliocentric longitude L0-L5, latitude
B0-B1 and radius R0-R4 terms [A, B, C], and the nutation arguments Y and
coefficients [a, b, c, d]), with the values the reference uses
(solweig_gpu/sun_position.py:202-477, 575-720), so that sun positions agree
with it to the last bit.

    python solweig_project_b200/data/make_spa_terms.py --ref <reference checkout>

The tables are read as literals from the source file (parsed, not run).
"""
from __future__ import annotations

import argparse
import ast
import json
import os

NAMES = ("L0_terms", "L1_terms", "L2_terms", "L3_terms", "L4_terms", "L5_terms", "B0_terms", "B1_terms",
         "R0_terms", "R1_terms", "R2_terms", "R3_terms", "R4_terms", "Y_terms", "nutation_terms")


def _literal(node):
    """The list literal of `np.array([...])`, `np.atleast_2d([...])` or `[...]`."""
    if isinstance(node, ast.Call):
        return _literal(node.args[0])
    return ast.literal_eval(node)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SOLWEIG_REFERENCE"), help="reference checkout")
    args = ap.parse_args()
    if not args.ref:
        raise SystemExit("name the reference checkout with --ref or SOLWEIG_REFERENCE")
    src = open(os.path.join(args.ref, "solweig_gpu", "sun_position.py")).read()
    found = {}
    for node in ast.walk(ast.parse(src)):
        if isinstance(node, ast.Assign) and len(node.targets) == 1 and isinstance(node.targets[0], ast.Name):
            name = node.targets[0].id
            if name in NAMES and not (isinstance(node.value, ast.Call) and
                                      getattr(node.value.func, "attr", "") == "atleast_2d" and
                                      isinstance(node.value.args[0], ast.Name)):
                val = _literal(node.value)
                if val and not isinstance(val[0], list):
                    val = [val]
                found[name] = [[float(x) for x in row] for row in val]
    missing = [n for n in NAMES if n not in found]
    if missing:
        raise SystemExit(f"tables not found: {missing}")
    out = {"source": "Solar Position Algorithm periodic terms (Reda and Andreas 2004, NREL/TP-560-34302, "
                     "Tables A4.2-A4.3): heliocentric L0-L5, B0-B1, R0-R4 rows [A, B, C]; nutation arguments Y "
                     "(63 x 5) and coefficients [a, b, c, d] (63 x 4)"}
    out.update({n: found[n] for n in NAMES})
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "spa_terms.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=0)
    print(f"wrote {path}: " + ", ".join(f"{n} {len(found[n])}" for n in NAMES))


if __name__ == "__main__":
    main()
