"""Test configuration: package path, the ``gpu`` marker and fixture helpers."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "curved-boundary-vlbm_b200"))
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))
GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libcvlbm.so")


@pytest.fixture(scope="session")
def golden_dir() -> Path:
    return GOLDEN
