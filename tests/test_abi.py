"""The C-ABI library loads and exports every symbol that include/cvlbm.h declares.

Runs without a GPU: only dlopen and symbol lookup, no compute calls.
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "cvlbm.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cvlbm\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "cvlbm2d_run" in names and "cvlbm3d_run" in names
    assert len(names) >= 12


def test_library_exports_every_declared_symbol():
    from curved_lbm import _build, _native

    if not _native.lib_path().exists():
        try:
            _build.build()
        except Exception as exc:  # pragma: no cover - toolchain missing
            pytest.skip(f"cannot build libcvlbm.so here: {exc}")
    lib = ctypes.CDLL(str(_native.lib_path()))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_native.EXPORTED) <= set(declared_functions())
    lib.cvlbm_version.restype = ctypes.c_int
    assert lib.cvlbm_version() == 10000


def test_cpu_device_is_rejected():
    from curved_lbm import _native

    with pytest.raises(ValueError):
        _native.torch_device("cpu")


def test_struct_layouts_match_the_library():
    """The ctypes mirrors of the ABI structs have the library's sizes."""
    from curved_lbm import _build, _native

    if not _native.lib_path().exists():
        try:
            _build.build()
        except Exception as exc:  # pragma: no cover - toolchain missing
            pytest.skip(f"cannot build libcvlbm.so here: {exc}")
    lib = ctypes.CDLL(str(_native.lib_path()))
    lib.cvlbm_struct_size.restype = ctypes.c_int64
    lib.cvlbm_struct_size.argtypes = [ctypes.c_int32]
    mirrors = (_native.Problem2D, _native.Fields2D, _native.Problem3D, _native.Fields3D,
               _native.StencilInput3D)
    for which, cls in enumerate(mirrors):
        assert lib.cvlbm_struct_size(which) == ctypes.sizeof(cls), cls.__name__
    assert lib.cvlbm_struct_size(7) == -1
