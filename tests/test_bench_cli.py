"""bench.py's reference arm, as the driver launches it, on the CPU.

`--impl reference` times the oracle on the host cores: one JSON line with the
contract's keys, warm-up and timed bench steps as asked, and an
`unavailable` line for a workload without a host implementation.
"""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _run(*args):
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_reference_arm_line():
    d = _run("--impl", "reference", "--steps", "2", "--warmup", "3", "--ref-step-seconds", "0.05")
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "cpu_baseline", "e2e", "config"):
        assert key in d, key
    assert d["impl"] == "reference" and d["metric"] == "MLUPS FP64" and d["unit"] == "MLUPS"
    assert d["steps"] == 2 and d["warmup"] == 3 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["config"]["workload"] == "annulus512"


def test_reference_arm_without_host_path():
    d = _run("--impl", "reference", "--workload", "gemm_bf16")
    assert d["impl"] == "reference" and "unavailable" in d
