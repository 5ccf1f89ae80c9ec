#!/usr/bin/env python3
"""Throughput benchmark of the curved-boundary VLBM time step on B200.

Metric: MLUPS (million active-node updates per second, FP64), reported as
an absolute figure and as a fraction of the measured HBM roofline.

Workloads (synthetic, seeded geometry; no external data):
  annulus512  D2Q4x6 traction annulus, 512^2 lattice on [0,1.1]^2, inner
              r=0.25 clamped, outer r=0.5 radial nominal traction ramped
              linearly 0 -> 0.05 over 20000 steps (then held); c=10,
              omega=1.8, alpha_u=0.85, theta_F=0.5, w_D=100, gamma=10,
              neo-Hooke mu=1, lambda=1; local_f closure, one displacement
              sweep and one F repair per step.  (Default.)
  shell192    D3Q6x12 spherical shell, 192^3 lattice on [0,2.2]^3, inner
              r=0.5 clamped, outer r=1.0 radial traction ramped 0 -> 0.05
              over 10000 steps; same physical parameters.
  batch256    256 D2Q4x6 superellipse shells, lattices 96^2..512^2 (seeded),
              solved together to residual 1e-8 (see batch_bench).
  tube_warmstart  3-D tubes under end stretch and twist: solver-generated
              equilibria, surrogate training, warm vs cold time-to-residual
              (see warmstart_bench).
  gemm_bf16   the surrogate's tcgen05 BF16 GEMM on its spectral-transform
              shapes and two square shapes (see gemm_bench).

One bench step = `--inner` lattice time steps replayed from one CUDA graph.
L2 (126 MB) is flushed between bench steps, outside the timed events.

Multi-GPU: the single-domain workloads do not shard, so each rank advances
an independent replica (weak scaling, no collectives on the data path);
`value` is the sum over ranks divided by the slowest rank's device time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "curved-boundary-vlbm_b200"))
sys.path.insert(0, str(ROOT))

BYTES_PER_UPDATE = {"annulus512": 416.0, "shell192": 1200.0}
HBM_FALLBACK_GBS = 6650.0


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def build_annulus(device=None, n=512, oracle=False, threads=1, intervals=None):
    from curved_lbm import workloads

    geom, mat, spec, kw = workloads.annulus(n)
    if intervals is not None:  # profiler captures of the node kernel's parts
        kw = dict(kw, local_displacement_interval=intervals[0],
                  local_compatibility_interval=intervals[1])
    if oracle:
        from oracle.oracle import Oracle2D

        s = Oracle2D(geom, material=mat, boundary=spec, threads=threads, **kw)
    else:
        from curved_lbm.two_d import curved_boundary_warp as c2

        s = c2.WarpCurvedBoundaryLBM2D(geom, material=mat, boundary=spec, device=device, **kw)
    U, disp = workloads.annulus_initial_state(n)
    s.initialize_from_numpy(U=U, displacement=disp, init_order=2)
    return s, geom.n_active


def build_shell(device=None, n=192, oracle=False, threads=1):
    from curved_lbm import workloads

    geom, mat, spec, kw = workloads.shell(n)
    if oracle:
        from oracle.oracle import Oracle3D

        s = Oracle3D(geom, material=mat, boundary=spec, threads=threads, **kw)
        s.initialize_identity()
        return s, s.N
    from curved_lbm.three_d import curved_boundary_warp3d as c3

    s = c3.WarpSparseCurvedBoundaryLBM3D(geom, material=mat, boundary=spec, device=device, **kw)
    return s, s.n_active


BUILDERS = {"annulus512": build_annulus, "shell192": build_shell}


def warmstart_bench(args, dev):
    """tube_warmstart: time-to-residual 1e-8 of 3-D tube solves, warm vs cold.

    Generates `--train` tube equilibria with the solver itself (cold starts to
    the tolerance, `--gen-batch` solves side by side), trains the FNO
    surrogate on the GPU (tensor-core spectral transforms), then solves
    `--test` held-out cases from the cold start (undeformed, end load ramped)
    and from the surrogate's prediction (end load at once).  `value` is the
    wall time of the cold-started plain solves (one after another) over that
    of the warm-started batched solves (every held-out case side by side);
    the report also holds warm plain and cold batched, so the warm-start and
    batching factors read separately.  Both starts reach the residual with
    their final errors against the converged FP64 field reported per case.
    """
    from curved_lbm import warmstart

    rep = warmstart.train_and_compare(nxy=args.tube_nxy, n_train=args.train, n_test=args.test,
                                      epochs=args.epochs, tol=args.tol, seed=7,
                                      device=str(dev), gen_batch=args.gen_batch,
                                      consecutive=args.consecutive)
    if args.rank != 0:
        return 0
    line = {"metric": "time-to-residual 1e-8, cold plain / warm batched",
            "value": rep["speedup_batched"],
            "unit": "x", "higher_is_better": True, "n_gpus": args.world, "dtype": "f64 solver, bf16 "
            "tensor-core surrogate (fp32 accumulate)", "data": "synthetic (solver-generated)",
            "config": {"workload": "tube_warmstart",
                       "lattice": [args.tube_nxy, args.tube_nxy, 2 * args.tube_nxy],
                       "train_cases": args.train, "test_cases": args.test,
                       "parallelism": f"training data-parallel over {args.world} rank(s); "
                                      "held-out comparison on rank 0",
                       "epochs": args.epochs, "tol": args.tol},
            "warm_plain_speedup": rep["speedup_wall"], "steps_ratio": rep["speedup_steps"],
            "equal_error_speedup": rep["speedup_batched_equal_error"],
            "equal_error_steps_ratio": rep["speedup_steps_equal_error"],
            "report": rep}
    print(json.dumps(line, default=float), flush=True)
    return 0


GEMM_SHAPES = ((128, 768, 65536), (128, 65536, 768), (1024, 1024, 8192), (4096, 4096, 4096))


def gemm_bench(args, dev):
    """gemm_bf16: the tcgen05 BF16 GEMM of the surrogate on the two FNO
    spectral-transform shapes of the 32 x 32 x 64 tube (128 rows, 768 modes,
    65,536 nodes) and two square shapes; CUDA events around 20 calls after 3
    warm-ups, inputs resident.  `value` is the 4096^3 rate.  The loader is
    the library's default (TMA); CVLBM_GEMM_LOADER=threads selects the
    thread-loaded kernel."""
    import torch

    from curved_lbm import _native

    lib = _native.load()
    peaks, peak_kind = measured_peaks()
    out = {}
    for M, N, K in GEMM_SHAPES:
        g = torch.Generator(device=dev).manual_seed(M + N + K)
        A = torch.randn(M, K, device=dev, generator=g).to(torch.bfloat16)
        B = torch.randn(N, K, device=dev, generator=g).to(torch.bfloat16)
        C = torch.empty(M, N, device=dev)
        err = torch.zeros(1, dtype=torch.int32, device=dev)
        ws = torch.empty(int(lib.cvlbm_gemm_bf16_workspace(M, N, K)) // 4, device=dev)

        def call():
            _native.check(lib.cvlbm_gemm_bf16(
                _native.ptr(A), _native.ptr(B), _native.ptr(C), M, N, K, K, K, N, 0,
                _native.ptr(err), _native.ptr(ws), ws.numel() * 4, _native.stream_ptr(dev)),
                "cvlbm_gemm_bf16")

        for _ in range(3):
            call()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(20):
            call()
        e1.record()
        e1.synchronize()
        us = e0.elapsed_time(e1) * 1e3 / 20
        out[f"{M}x{N}x{K}"] = {"us": round(us, 1), "tflops": round(2.0 * M * N * K / us / 1e6, 1),
                               "error_flag": int(err.item())}
    top = out["4096x4096x4096"]["tflops"]
    line = {"metric": "bf16 GEMM TFLOP/s (tcgen05, fp32 accumulate)", "value": top,
            "unit": "TFLOP/s", "higher_is_better": True, "n_gpus": 1, "dtype": "bf16",
            "data": "synthetic", "loader": os.environ.get("CVLBM_GEMM_LOADER", "tma"),
            "config": {"workload": "gemm_bf16", "shapes": out},
            "roofline": {"bound": "tensor", "achieved": top,
                         "peak": peaks.get("bf16_tflops"), "peak_kind": peak_kind,
                         "unit": "TFLOP/s",
                         "frac": top / peaks["bf16_tflops"] if peaks.get("bf16_tflops") else None}}
    print(json.dumps(line), flush=True)
    return 0


def batch_bench(args, dev):
    """batch256: 256 superellipse shells (96^2..512^2) to residual 1e-8.

    The solvers start undeformed; the timed region is the whole batched solve
    (graph replays of `--inner` lattice steps with a residual check every 100
    steps) until every instance has retired.  One bench step = one replay.
    `value` = active-node updates of all instances / device time of the solve.
    Under torchrun the instances are dealt round-robin to the ranks (no
    exchange between ranks); times are the max over ranks.
    """
    import torch

    from curved_lbm import _native, replicas, workloads
    from curved_lbm.batch import BatchedCurvedBoundaryLBM2D

    n_inst = args.instances
    world, rank = args.world, args.rank
    t0 = time.perf_counter()
    params = replicas.deal(workloads.superellipse_params(n_inst), rank, world)
    geoms = workloads.superellipse_geometries(
        params, processes=max(1, (os.cpu_count() or 1) // world))
    geom_s = time.perf_counter() - t0
    solvers = workloads.superellipse_solvers(params, geoms, device=str(dev))
    setup_s = time.perf_counter() - t0
    batch = BatchedCurvedBoundaryLBM2D(solvers)
    tuned = batch.autotune(steps=4)
    active = np.array([s.geometry.n_active for s in solvers], dtype=np.float64)
    stream = torch.cuda.current_stream(dev)
    n0 = _native.launch_count()
    g = batch.graph(args.inner, check_every=100, tol=args.tol,
                    t_min=workloads.SUPERELLIPSE_RAMP_TIME)
    per_graph = _native.launch_count() - n0
    replays, device_ms = 0, 0.0
    st0 = batch.status()
    with ClockSampler(args.local) as clocks:
        torch.cuda.synchronize(dev)
        w0 = time.perf_counter()
        st = st0
        while st["active"].any() and replays < args.max_replays:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.launch(g)
            e1.record(stream)
            st = batch.status()
            device_ms += e0.elapsed_time(e1)
            replays += 1
        wall_s = time.perf_counter() - w0
    steps = st["steps"] - st0["steps"]
    updates = float((active * steps).sum())
    ng, nw = batch.launch_grid()
    n_conv, n_bad = int((st["status"] == 1).sum()), int((st["status"] == -1).sum())
    # instance numbers (in the seeded table) of the instances that went invalid
    mine = replicas.deal(list(range(n_inst)), rank, world)
    bad_ids = [[int(mine[k]), int(st["steps"][k])] for k in np.flatnonzero(st["status"] == -1)]
    (device_ms, wall_s), (updates, n_conv, n_bad) = replicas.reduce_times_and_counts(
        [device_ms, wall_s], [updates, n_conv, n_bad], device=dev)
    n_conv, n_bad = int(n_conv), int(n_bad)
    if rank != 0:
        return 0
    sum_n2 = int(sum(p["n"] ** 2 for p in workloads.superellipse_params(n_inst)))
    line = {
        "metric": "MLUPS FP64", "value": updates / (device_ms * 1e-3) / 1e6, "unit": "MLUPS",
        "n_gpus": world, "steps": replays, "warmup": 0,
        "ms_per_step": device_ms / max(replays, 1),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "batch256", "instances": n_inst,
                   "parallelism": f"instances dealt over {world} rank(s)",
                   "lattice_steps_per_bench_step": args.inner,
                   "active_nodes_rank0": int(active.sum()), "sum_n2": sum_n2,
                   "tile_variant": batch.tile_variant,
                   "autotune_ms_per_step": {str(k): round(v, 4) for k, v in tuned.items()},
                   "persistent_node_grid": ng, "work_items": nw,
                   "residual": "|u-u_prev|_2/(100 |u|_2) over active nodes, checked every 100 steps "
                               f"after t >= {workloads.SUPERELLIPSE_RAMP_TIME}",
                   "tol": args.tol, "host_setup_s": round(setup_s, 1), "host_geometry_s": round(geom_s, 1),
                   "l2": "working set (%.1f GB of populations) far above L2"
                         % (sum_n2 * 24 * 8 * 2 / 1e9)},
        "time_to_residual_s": {"device": device_ms * 1e-3, "wall": wall_s},
        "instances_converged": n_conv, "instances_invalid": n_bad,
        "invalid_instances_rank0": bad_ids,  # [instance number, step when retired]
        "steps_per_instance_rank0": {"min": int(steps.min()), "max": int(steps.max()),
                                     "mean": float(steps.mean())},
        "clocks": clocks.summary(),
        "gpu_launches": int(per_graph * replays),
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# measurement helpers
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region starts once the sampler reports (bounded wait)
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.rows.clear()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 9
                          for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def measured_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            return json.loads(path.read_text()), "measured"
        except Exception:
            pass
    return {"hbm_gbs": HBM_FALLBACK_GBS}, "fallback"


def ncu_traffic(workload: str):
    """(DRAM bytes per launch of the bracketed node kernels, where they come from),
    read from the committed ncu summary figures."""
    path = ROOT / "profiles" / "traffic.json"
    if not path.exists():
        return None, None
    try:
        ent = json.loads(path.read_text()).get(workload) or {}
        return ent.get("bytes"), ent.get("source")
    except Exception:
        return None, None


def cpu_baseline(workload: str, seconds: float, threads: int):
    """Oracle (C port of the reference kernels) on the host cores: lattice steps
    of the workload in chunks of 5 until `seconds` of CPU time have passed."""
    from oracle import oracle as orc

    orc.load()
    builder = BUILDERS[workload]
    s, n_active = builder(oracle=True, threads=threads)
    s.step()  # warm the page cache and OpenMP pool
    steps = 0
    t0 = time.perf_counter()
    while True:
        for _ in range(5):
            s.step()
        steps += 5
        dt = time.perf_counter() - t0
        if dt >= seconds:
            break
    return {"value": n_active * steps / dt / 1e6, "unit": "MLUPS", "cores": threads,
            "kind": "port",
            "sample": f"{steps} lattice time steps of {workload} ({n_active} active nodes), "
                      f"oracle/cvlbm_oracle.c, OpenMP {threads} threads, {dt:.1f} s"}


# ---------------------------------------------------------------------------
def init_dist():
    from curved_lbm import replicas

    return replicas.init(timeout_s=600.0)


def reference_arm(args, world, rank):
    """`--impl reference`: the reference's kernels on the host cores (the
    oracle, a C port pinned to the reference's own outputs; Warp cannot be
    installed here).  Rank 0 alone runs: `--warmup` untimed and `--steps`
    timed bench steps, each a bounded sample of `chunk` lattice steps of the
    same workload, sized to about `--ref-step-seconds` of host time."""
    if rank != 0:
        return 0
    if args.workload not in BUILDERS:
        print(json.dumps({"impl": "reference", "unavailable":
                          f"no host implementation of the {args.workload} workload"}), flush=True)
        return 0
    from oracle import oracle as orc

    orc.load()
    threads = os.cpu_count() or 1
    s, n_active = BUILDERS[args.workload](oracle=True, threads=threads)
    s.step()  # page cache and OpenMP pool
    t0 = time.perf_counter()
    s.step()
    one = time.perf_counter() - t0
    chunk = max(1, min(args.inner, int(round(args.ref_step_seconds / max(one, 1e-9)))))
    for _ in range(args.warmup):
        for _ in range(chunk):
            s.step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for _ in range(chunk):
            s.step()
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = n_active * chunk * args.steps / total / 1e6
    sample = (f"{args.steps} bench steps of {chunk} lattice time steps of {args.workload} "
              f"({n_active} active nodes), oracle/cvlbm_oracle.c, OpenMP {threads} threads, "
              f"{total:.1f} s")
    line = {
        "impl": "reference", "metric": "MLUPS FP64", "value": value, "unit": "MLUPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "lbm_steps_per_bench_step": chunk},
        "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "reference Warp 1.10.1 is not installable here (no wheel, no network); the "
                "reference arm times oracle/cvlbm_oracle.c, a C port of its kernels pinned "
                "to its own outputs",
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="annulus512",
                    choices=sorted(BUILDERS) + ["batch256", "tube_warmstart", "gemm_bf16"])
    ap.add_argument("--tube-nxy", type=int, default=32, help="tube_warmstart: lattice nx = ny")
    ap.add_argument("--train", type=int, default=256, help="tube_warmstart: training cases")
    ap.add_argument("--test", type=int, default=4, help="tube_warmstart: held-out cases")
    ap.add_argument("--epochs", type=int, default=300, help="tube_warmstart: training epochs")
    ap.add_argument("--gen-batch", type=int, default=32,
                    help="tube_warmstart: training solves run side by side")
    ap.add_argument("--consecutive", type=int, default=1,
                    help="tube_warmstart: residual checks in a row below the tolerance")
    ap.add_argument("--instances", type=int, default=256, help="batch256: instance count")
    ap.add_argument("--tol", type=float, default=1e-8, help="batch256: residual tolerance")
    ap.add_argument("--max-replays", type=int, default=100000, help="batch256: replay cap")
    ap.add_argument("--inner", type=int, default=100, help="lattice steps per bench step")
    ap.add_argument("--local-intervals", default="",
                    help="annulus: 'SWEEP,REPAIR' step intervals of the displacement sweep and "
                         "the F repair (0 = off), for profiler captures of the node kernel's "
                         "parts, not bench lines")
    ap.add_argument("--size", type=int, default=0,
                    help="lattice nodes per axis (0 = the workload's own size; smaller sizes "
                         "are for profiler captures, not bench lines)")
    ap.add_argument("--ref-step-seconds", type=float, default=0.5,
                    help="--impl reference: host time of one bench step (sizes the sample)")
    ap.add_argument("--ref-seconds", type=float, default=12.0,
                    help="CPU time of the oracle sample (CPU baseline and reference arm)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--overlap", default="default", choices=["default", "on", "off"],
                    help="link-kernel overlap of the fused step (default: the solver's)")
    ap.add_argument("--tile-variant", type=int, default=-1,
                    help="fused 2-D tile shape or 3-D collide variant; -1 = autotune")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.inner % 2:
        args.inner += 1
    world, rank, local = init_dist()
    if args.impl == "reference":
        rc = reference_arm(args, world, rank)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return rc

    import torch

    from curved_lbm import _native

    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    args.local, args.world, args.rank = local, world, rank
    if args.workload == "gemm_bf16":
        rc = gemm_bench(args, dev) if rank == 0 else 0
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return rc
    if args.workload == "tube_warmstart":
        # equilibria generated and the surrogate trained data-parallel over
        # the ranks; the held-out warm / cold comparison runs on rank 0
        rc = warmstart_bench(args, dev)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return rc
    if args.workload == "batch256":
        if args.inner == 100:
            args.inner = 1000
        rc = batch_bench(args, dev)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return rc
    size_kw = {"n": args.size} if args.size > 0 else {}
    if args.local_intervals:
        if args.workload != "annulus512":
            raise SystemExit("--local-intervals applies to the annulus workload only")
        size_kw["intervals"] = tuple(int(v) for v in args.local_intervals.split(","))
    solver, n_active = BUILDERS[args.workload](device=str(dev), **size_kw)
    if args.overlap != "default" and hasattr(solver, "overlap_links"):
        solver.overlap_links = args.overlap == "on"
    tuned = {}
    if hasattr(solver, "autotune"):
        if args.tile_variant >= 0:
            solver._select_variant(args.tile_variant)
        else:
            tuned = solver.autotune()
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)

    # With the link kernel overlapped by the next step's inner tiles, the node
    # kernel runs as two launches on two streams; its duration alone is then
    # timed afterwards on a graph of the same steps without the overlap.
    overlap = bool(getattr(solver, "overlap_links", False))
    timer = _native.KernelTimer(args.inner)
    # the 2-D cut-link kernel's own event pairs (timed where the node kernel is)
    ltimer = _native.KernelTimer(args.inner, "links") if args.workload == "annulus512" else None
    if not overlap:
        timer.attach()
        if ltimer:
            ltimer.attach()
    n0 = _native.launch_count()
    graph = solver.capture_graph(args.inner)
    launches_per_graph = _native.launch_count() - n0
    if not overlap:
        timer.detach()
        if ltimer:
            ltimer.detach()

    for _ in range(args.warmup):
        graph.launch()
    torch.cuda.synchronize(dev)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()

    step_ms, kern_ms, kern_n = [], 0.0, 0
    link_ms, link_n = 0.0, 0
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            graph.launch()
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            if not overlap:
                ms, cnt = timer.elapsed()
                kern_ms += ms
                kern_n += cnt
                if ltimer:
                    ms, cnt = ltimer.elapsed()
                    link_ms += ms
                    link_n += cnt
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
    kern_total_ms = float(sum(step_ms))
    if overlap:
        solver.overlap_links = False
        timer.attach()
        if ltimer:
            ltimer.attach()
        kgraph = solver.capture_graph(args.inner)
        timer.detach()
        if ltimer:
            ltimer.detach()
        solver.overlap_links = True
        for _ in range(2):
            kgraph.launch()
        timer.elapsed()
        if ltimer:
            ltimer.elapsed()
        kern_total_ms = 0.0
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            kgraph.launch()
            e1.record(stream)
            e1.synchronize()
            kern_total_ms += e0.elapsed_time(e1)
            ms, cnt = timer.elapsed()
            kern_ms += ms
            kern_n += cnt
            if ltimer:
                ms, cnt = ltimer.elapsed()
                link_ms += ms
                link_n += cnt
        del kgraph
    total_ms = float(sum(step_ms))
    from curved_lbm import replicas

    (total_ms,), _ = replicas.reduce_times_and_counts([total_ms], [], device=dev)
    updates = float(n_active) * args.inner * args.steps * world
    value = updates / (total_ms * 1e-3) / 1e6

    # end to end through the public API: pinned host traction -> device,
    # lattice steps, invalid/finite check read back to the host
    e2e = None
    if hasattr(solver, "enable_dynamic_link_traction"):
        nl = solver.geometry.n_links
        hx = torch.empty(nl, dtype=torch.float64).pin_memory()
        hy = torch.empty(nl, dtype=torch.float64).pin_memory()
        nxv = torch.as_tensor(solver.geometry.link_nx)
        nyv = torch.as_tensor(solver.geometry.link_ny)
        out = torch.empty(2, dtype=torch.float64).pin_memory()
        amp, ramp = solver.boundary_params[0], solver.boundary_params[1]
        outer = torch.as_tensor(solver.geometry.link_boundary_id == 1)

        def upload():
            # the workload's own load (radial traction ramped over ramp_time),
            # computed on the host at the middle of the step chunk about to run
            tm = solver.time + 0.5 * args.inner * solver.dt
            sc = min(tm / ramp, 1.0) if ramp > 0 else 1.0
            hx.copy_(torch.where(outer, amp * sc * nxv, torch.zeros_like(nxv)))
            hy.copy_(torch.where(outer, amp * sc * nyv, torch.zeros_like(nyv)))
            solver.link_traction_x.copy_(hx, non_blocking=True)
            solver.link_traction_y.copy_(hy, non_blocking=True)

        def readback():
            vmax = torch.stack([solver.invalid.double().max(), solver.U[:2].abs().max()])
            out.copy_(vmax, non_blocking=True)
            torch.cuda.synchronize(dev)

        # one untimed iteration: run() caches its CUDA graph and the read-back's
        # kernels load on first use
        upload()
        solver.enable_dynamic_link_traction(True)
        solver.run(args.inner)
        readback()
        # L2 flushed between steps as for `value` (outside the timed region):
        # without it the populations stay in L2 from one bench step to the next
        e2e_s = 0.0
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            upload()
            solver.run(args.inner)
            readback()
            e2e_s += time.perf_counter() - t0
        solver.enable_dynamic_link_traction(False)
        e2e = {"value": float(n_active) * args.inner * args.steps * world / e2e_s / 1e6,
               "unit": "MLUPS", "h2d_bytes_per_step": int(2 * nl * 8),
               "d2h_bytes_per_step": 16,
               "path": "WarpCurvedBoundaryLBM2D.run() with dynamic link traction uploaded "
                       "from pinned host memory each bench step; max|v| and the invalid "
                       "flag read back; L2 flushed between bench steps"}

    peaks, peak_kind = measured_peaks()
    avg_kern_s = kern_ms * 1e-3 / max(kern_n, 1)
    algo_bytes = n_active * BYTES_PER_UPDATE[args.workload]
    achieved = algo_bytes / avg_kern_s / 1e9 if kern_n else None
    traffic, traffic_src = ncu_traffic(args.workload)
    roofline = {"bound": "hbm", "kernel": "bulk node kernel (bracketed per lattice step)",
                "achieved": achieved, "peak": peaks.get("hbm_gbs", HBM_FALLBACK_GBS),
                "peak_kind": peak_kind, "unit": "GB/s",
                "frac": (achieved / peaks.get("hbm_gbs", HBM_FALLBACK_GBS)) if achieved else None,
                "traffic": traffic, "traffic_source": traffic_src,
                "algorithmic_bytes_per_launch": algo_bytes,
                "avg_launch_ms": avg_kern_s * 1e3,
                "step_frac": (kern_ms / kern_total_ms) if kern_total_ms else None,
                "timed_without_overlap": overlap,
                "whole_step_achieved": updates / world * BYTES_PER_UPDATE[args.workload]
                / (total_ms * 1e-3) / 1e9}
    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            base = cpu_baseline(args.workload, args.ref_seconds, os.cpu_count() or 1)
        except Exception as exc:  # the oracle is optional for the GPU number
            base = {"value": None, "unit": "MLUPS", "cores": 0, "kind": "port",
                    "sample": f"unavailable: {exc}"}
    line = {
        "metric": "MLUPS FP64", "value": value, "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "n_active": int(n_active),
                   "lbm_steps_per_bench_step": args.inner,
                   "l2": "flushed between bench steps (256 MB write)",
                   "parallelism": f"replicas x{world}",
                   "tile_variant": getattr(solver, "tile_variant", None),
                   "node_variant": getattr(solver, "node_variant", None),
                   "overlap_links": overlap,
                   "autotune_us_per_step": {str(k): round(v, 2) for k, v in tuned.items()}},
        "e2e": e2e, "roofline": roofline, "cpu_baseline": base,
        "clocks": clocks.summary(),
        "gpu_launches": int(launches_per_graph * args.steps),
    }
    if link_n:
        # the same kernel launched eagerly (no graph): event pairs around each
        # launch on the stream, without the graph's event-node transitions
        eager_ms, eager_n = 0.0, 0
        if hasattr(solver, "use_graphs"):
            use_graphs, ov = solver.use_graphs, solver.overlap_links
            solver.use_graphs, solver.overlap_links = False, False
            ltimer.reset()
            ltimer.attach()
            for _ in range(args.steps):
                flush.zero_()
                solver.run(args.inner)
                ms, cnt = ltimer.elapsed()
                ltimer.reset()
                eager_ms += ms
                eager_n += cnt
            ltimer.detach()
            solver.use_graphs, solver.overlap_links = use_graphs, ov
        line["link_kernel"] = {
            "avg_us": link_ms * 1e3 / link_n, "launches": link_n,
            "timed": "CUDA events around each cut-link kernel launch, in the graph without "
                     "the link overlap (L2 flushed between bench steps)",
            "eager_avg_us": eager_ms * 1e3 / eager_n if eager_n else None,
            "eager_timed": "the same, launched without a graph (one native call per bench "
                           "step)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del graph
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
