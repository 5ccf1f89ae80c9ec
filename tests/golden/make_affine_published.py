#!/usr/bin/env python3
"""Extract the reference's published affine-annulus convergence rows.

The reference records, per grid n, the relative L2 errors of its affine
Dirichlet annulus against the exact solution (cases/affine_annulus.py) in
``validation/release_verification.json`` (full_benchmark_verification ->
cases -> affine_annulus -> rows).  This script copies those numbers, and only
those, into ``affine_published.json`` beside it::

    python tests/golden/make_affine_published.py --ref <reference checkout>

(or set CVLBM_REFERENCE_ROOT instead of passing --ref).
"""

from __future__ import annotations

import argparse
import json
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
METRICS = ("rel_l2_u", "rel_l2_v", "rel_l2_F", "rel_l2_F_minus_I", "rel_l2_sigma", "min_J", "max_J")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("CVLBM_REFERENCE_ROOT"),
                    help="root of the reference checkout (or CVLBM_REFERENCE_ROOT)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("--ref (or CVLBM_REFERENCE_ROOT) is required")
    src = Path(args.ref) / "validation" / "release_verification.json"
    data = json.loads(src.read_text())
    rows = data["full_benchmark_verification"]["cases"]["affine_annulus"]["rows"]
    out = {"source": "validation/release_verification.json: full_benchmark_verification."
                     "cases.affine_annulus.rows",
           "rows": [{"n": int(r["n"]), "steps": int(r["steps"]), "time": float(r["time"]),
                     **{m: float(r["metrics"][m]["value"]) for m in METRICS}} for r in rows]}
    (HERE / "affine_published.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"{len(out['rows'])} rows")


if __name__ == "__main__":
    main()
