#!/usr/bin/env python3
"""Replay batched superellipse instances on the oracle -- TEST INFRASTRUCTURE.

The batched benchmark retires an instance with status -1 when its Jacobian
turns non-positive.  This script answers whether the reference's arithmetic
(the oracle, pinned to the reference's fixtures) does the same on those
instances: it runs each listed instance of the seeded table
(curved_lbm.workloads.superellipse_params) from the undeformed state and
reports the first check (every `--every` steps) at which the oracle's state
is invalid (the reference's `invalid_state`: flag set, or U not finite), or
that it stayed valid for `--steps` steps.

    python oracle/replay_instances.py --ids 3,17:900,42 [--steps 2000] [--procs 4]

(`id:steps` sets that instance's own step limit.)

Prints one JSON line per instance and a summary line.
"""

from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _paths():
    for p in (str(ROOT / "curved-boundary-vlbm_b200"), str(ROOT)):
        if p not in sys.path:
            sys.path.insert(0, p)


def replay(args):
    idx, steps, every, threads, n_inst = args
    _paths()
    import numpy as np

    from curved_lbm import workloads
    from oracle.oracle import Oracle2D

    prm = workloads.superellipse_params(n_inst)[idx]
    t0 = time.time()
    geom = workloads.superellipse_geometry(prm)
    mat, spec, kw = workloads.superellipse_case(prm)
    o = Oracle2D(geom, material=mat, boundary=spec, threads=threads, **kw)
    U, disp = workloads.annulus_initial_state(prm["n"])
    o.initialize_from_numpy(U=U, displacement=disp, init_order=2)
    act = geom.active.astype(bool)
    bad_at = None
    vmax = 0.0
    while o.steps < steps:
        o.run(min(every, steps - o.steps))
        o.refresh()
        vmax = float(np.max(np.abs(o.U[:2, act]))) if act.any() else 0.0
        if int(o.invalid[0]) != 0 or not np.isfinite(o.U[:, act]).all():
            bad_at = o.steps
            break
    return {"instance": idx, "n": prm["n"], "p": prm["p"], "a": prm["a"], "b": prm["b"],
            "r_in": prm["r_in"], "traction": prm["traction"], "steps_run": o.steps,
            "invalid_at_step": bad_at, "max_abs_v": vmax if math.isfinite(vmax) else None,
            "seconds": round(time.time() - t0, 1)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ids", required=True,
                    help="comma-separated instance numbers, each optionally id:steps")
    ap.add_argument("--instances", type=int, default=256, help="size of the seeded table")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--procs", type=int, default=max(1, (os.cpu_count() or 1) // 2))
    a = ap.parse_args()
    ids = []
    for v in a.ids.split(","):
        if v.strip():
            i, _, st = v.partition(":")
            ids.append((int(i), int(st) if st else a.steps))
    threads = max(1, (os.cpu_count() or 1) // max(1, a.procs))
    jobs = [(i, st, a.every, threads, a.instances) for i, st in ids]
    with mp.get_context("spawn").Pool(a.procs) as pool:
        out = []
        for r in pool.imap_unordered(replay, jobs):
            print(json.dumps(r), flush=True)
            out.append(r)
    bad = sorted(r["instance"] for r in out if r["invalid_at_step"] is not None)
    print(json.dumps({"replayed": len(out), "invalid_on_oracle": len(bad), "invalid_ids": bad}))


if __name__ == "__main__":
    main()
