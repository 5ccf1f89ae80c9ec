"""ctypes binding of libcvlbm.so (declared in ``include/cvlbm.h``).

The solver classes keep their state in PyTorch CUDA tensors and hand raw
device pointers to the library; the library launches the sm_100a kernels on
PyTorch's current stream.  There is no CPU or fallback path: importing a
solver on a machine without the built library or without a CUDA device
raises immediately.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libcvlbm.so"
_lib = None

i32 = C.c_int32
i64 = C.c_int64
f64 = C.c_double
pI = C.c_void_p  # device pointers are passed as opaque addresses


class Material(C.Structure):
    _fields_ = [("model", i32), ("reserved", i32), ("lam", f64), ("mu", f64), ("p0", f64),
                ("p1", f64), ("p2", f64), ("j_floor", f64)]


class Problem2D(C.Structure):
    _fields_ = [
        ("nx", i32), ("ny", i32), ("n_links", i32), ("recon", i32), ("normal_solver", i32),
        ("source_mode", i32),
        ("dx", f64), ("dy", f64), ("dt", f64), ("omega", f64), ("c", f64),
        ("source", f64 * 6),
        ("mat", Material),
        ("disp_interval", i32), ("disp_sweeps", i32), ("disp_bid", i32), ("rep_interval", i32),
        ("interior_only", i32), ("use_dynamic_traction", i32),
        ("relax", f64), ("weight", f64), ("blend", f64),
        ("active", pI),
        ("link_i", pI), ("link_j", pI), ("link_q", pI), ("link_bid", pI),
        ("link_eta", pI), ("link_xb", pI), ("link_yb", pI), ("link_nx", pI), ("link_ny", pI),
        ("lsq_i", pI), ("lsq_j", pI),
        ("lsq_wb", pI), ("lsq_wt", pI), ("lsq_wx", pI), ("lsq_wy", pI),
        ("lsq_valid", pI),
        ("node_link_start", pI), ("node_link_list", pI),
        ("bc_kind", pI), ("bc_mode", pI), ("bc_params", pI),
        ("traction_x", pI), ("traction_y", pI),
        ("tiles", pI), ("n_tiles", i32), ("tiles_j", i32), ("need_fields", pI),
        ("link_partner", pI), ("lsq_node", pI), ("link_order", pI),
        ("tile_variant", i32), ("tile_i", i32), ("n_tiles_inner", i32), ("overlap", i32),
        ("link_rows", pI), ("lsq_node_slot", pI), ("lsq_wb_slot", pI), ("lsq_wt_slot", pI),
        ("lsq_wx_slot", pI), ("lsq_wy_slot", pI),
        ("collision_model", i32), ("ghost_omega", f64), ("kinetic_filter", f64),
    ]


def link_row2_dtype():
    """cvlbm2d_link_row (96 bytes) as a NumPy record."""
    import numpy as np

    return np.dtype({"names": ["ell", "node", "upstream", "q", "bid", "lsq_valid", "i", "j",
                               "eta", "xb", "yb", "nx", "ny"],
                     "formats": ["<i4"] * 8 + ["<f8"] * 5,
                     "offsets": [0, 4, 8, 12, 16, 20, 24, 28, 32, 40, 48, 56, 64],
                     "itemsize": 96})


class Fields2D(C.Structure):
    _fields_ = [(name, pI) for name in
                ("f0", "f1", "fpost", "U", "u", "u_next", "u_star", "P", "sigma", "invalid",
                 "clock", "link_scratch")]


class Problem3D(C.Structure):
    _fields_ = [
        ("n_active", i32), ("n_links", i32), ("nx", i32), ("ny", i32), ("nz", i32),
        ("recon", i32), ("normal_solver", i32), ("source_mode", i32), ("has_char", i32),
        ("has_tangent_lsq", i32),
        ("disp_interval", i32), ("disp_sweeps", i32), ("disp_bid", i32), ("rep_interval", i32),
        ("dx", f64), ("dy", f64), ("dz", f64), ("dt", f64), ("omega", f64), ("c", f64),
        ("source", f64 * 12),
        ("mat", Material),
        ("relax", f64), ("weight", f64), ("blend", f64),
        ("active_i", pI), ("active_j", pI), ("active_k", pI),
        ("neighbor", pI),
        ("link_p", pI), ("link_up", pI), ("link_q", pI), ("link_bid", pI),
        ("link_eta", pI), ("link_xb", pI), ("link_yb", pI), ("link_zb", pI),
        ("link_nx", pI), ("link_ny", pI), ("link_nz", pI),
        ("lsq_p", pI), ("lsq_wt1", pI), ("lsq_wt2", pI), ("lsq_valid", pI),
        ("char_idx", pI), ("char_w", pI),
        ("node_link_start", pI), ("node_link_list", pI),
        ("bc_kind", pI), ("bc_mode", pI), ("bc_comp_kind", pI), ("bc_params", pI),
        ("dyn_enabled", pI), ("dyn_traction", pI),
        ("need_slot", pI), ("n_need", i32), ("node_variant", i32), ("char_slot", pI),
        ("link_partner", pI), ("link_order", pI), ("link_nodes", pI), ("n_link_nodes", i32),
        ("overlap", i32),
        ("wave_items", pI), ("n_wave_items", i32), ("n_planes", i32), ("wave_plane_chunks", pI),
        ("char_slot_lm", pI), ("char_w_lm", pI),
    ]


class Fields3D(C.Structure):
    _fields_ = [(name, pI) for name in
                ("f0", "f1", "U", "u", "u_next", "u_star", "link_kind", "link_comp_kind",
                 "link_bv", "link_Fb", "link_Pb", "char_state", "invalid", "clock",
                 "link_scratch", "U_need", "wave_sync")]


class StencilInput3D(C.Structure):
    _fields_ = [("nx", i32), ("ny", i32), ("nz", i32), ("n_links", i32), ("dx", f64),
                ("active_id", pI)] + [(name, pI) for name in (
                    "link_i", "link_j", "link_k", "link_q", "link_eta", "link_xb", "link_yb",
                    "link_zb", "link_nx", "link_ny", "link_nz", "link_mask")]


EXPORTED = (
    "cvlbm2d_run",
    "cvlbm2d_apply_boundary",
    "cvlbm2d_refresh",
    "cvlbm2d_stress",
    "cvlbm2d_kinetic_filter",
    "cvlbm2d_init_populations",
    "cvlbm2d_init_work_bytes",
    "cvlbm_field_summary",
    "cvlbm_field_summary_work_bytes",
    "cvlbm3d_run",
    "cvlbm3d_apply_boundary",
    "cvlbm3d_refresh",
    "cvlbm3d_set_ustar",
    "cvlbm3d_build_char_stencil",
    "cvlbm2d_graph_create",
    "cvlbm3d_graph_create",
    "cvlbm_graph_launch",
    "cvlbm_graph_destroy",
    "cvlbm_version",
    "cvlbm_struct_size",
    "cvlbm_last_error",
    "cvlbm_timer_create",
    "cvlbm_timer_destroy",
    "cvlbm_timer_reset",
    "cvlbm_timer_elapsed",
    "cvlbm_timer_attach",
    "cvlbm_timer_attach_links",
    "cvlbm_launch_count",
    "cvlbm2d_tile_variant",
    "cvlbm2d_run_static_scratch",
    "cvlbm2d_batch_create",
    "cvlbm2d_batch_run",
    "cvlbm2d_batch_graph_create",
    "cvlbm2d_batch_status",
    "cvlbm2d_batch_launch_grid",
    "cvlbm2d_batch_destroy",
    "cvlbm_gemm_bf16",
    "cvlbm_gemm_bf16_workspace",
    "cvlbm_fno_pointwise_fwd",
    "cvlbm_fno_gelu_bwd",
    "cvlbm_fno_pointwise_bwd",
    "cvlbm_fno_pointwise_scratch",
    "cvlbm_fno_spec_mix_fwd",
    "cvlbm_fno_spec_mix_bwd",
    "cvlbm_fno_to_bf16",
    "cvlbm_fno_mse",
    "cvlbm_fno_adam",
)


def lib_path() -> Path:
    return Path(os.environ.get("CVLBM_LIBRARY", str(_LIB_PATH)))


def load(require_cuda: bool = True):
    """Load libcvlbm.so and declare its signatures; raises if unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not path.exists():
        raise RuntimeError(
            f"libcvlbm.so not found at {path}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (nvcc, sm_100a)")
    lib = C.CDLL(str(path))
    P2, F2, P3, F3 = C.POINTER(Problem2D), C.POINTER(Fields2D), C.POINTER(Problem3D), C.POINTER(Fields3D)
    sig = {
        "cvlbm2d_run": (i32, [P2, F2, f64, i64, i32, i32, pI]),
        "cvlbm2d_apply_boundary": (i32, [P2, F2, f64, i32, pI]),
        "cvlbm2d_refresh": (i32, [P2, F2, pI]),
        "cvlbm2d_stress": (i32, [P2, F2, pI]),
        "cvlbm2d_kinetic_filter": (i32, [P2, F2, pI]),
        "cvlbm2d_init_populations": (i32, [P2, pI, i32, pI, pI, pI, pI]),
        "cvlbm2d_init_work_bytes": (i64, [i32, i32]),
        "cvlbm_field_summary": (i32, [i32, i64, pI, pI, pI, pI, C.POINTER(f64), pI]),
        "cvlbm_field_summary_work_bytes": (i64, []),
        "cvlbm3d_run": (i32, [P3, F3, f64, i64, i32, i32, pI]),
        "cvlbm3d_apply_boundary": (i32, [P3, F3, f64, i32, pI]),
        "cvlbm3d_refresh": (i32, [P3, F3, pI]),
        "cvlbm3d_set_ustar": (i32, [P3, F3, pI, pI]),
        "cvlbm3d_build_char_stencil": (i32, [C.POINTER(StencilInput3D), pI, pI, pI, pI, pI]),
        "cvlbm2d_graph_create": (i32, [P2, F2, i64, i32, C.POINTER(pI)]),
        "cvlbm3d_graph_create": (i32, [P3, F3, i64, i32, C.POINTER(pI)]),
        "cvlbm_graph_launch": (i32, [pI, pI]),
        "cvlbm_graph_destroy": (None, [pI]),
        "cvlbm_version": (i32, []),
        "cvlbm_struct_size": (C.c_int64, [i32]),
        "cvlbm_timer_create": (i32, [i32, C.POINTER(pI)]),
        "cvlbm_timer_destroy": (None, [pI]),
        "cvlbm_timer_reset": (i32, [pI]),
        "cvlbm_timer_elapsed": (i32, [pI, C.POINTER(f64), C.POINTER(i32)]),
        "cvlbm_timer_attach": (i32, [pI]),
        "cvlbm_timer_attach_links": (i32, [pI]),
        "cvlbm_launch_count": (i64, []),
        "cvlbm2d_tile_variant": (i32, [i32]),
        "cvlbm2d_run_static_scratch": (i32, [P2, F2, f64, i64, i32, pI]),
        "cvlbm_last_error": (C.c_char_p, []),
        "cvlbm2d_batch_create": (i32, [i32, P2, F2, C.POINTER(i64), C.POINTER(f64), i32, i32,
                                       C.POINTER(pI)]),
        "cvlbm2d_batch_run": (i32, [pI, i32, i32, f64, f64, pI]),
        "cvlbm2d_batch_graph_create": (i32, [pI, i32, i32, f64, f64, C.POINTER(pI)]),
        "cvlbm2d_batch_status": (i32, [pI, C.POINTER(i32), C.POINTER(i32), C.POINTER(i64),
                                       C.POINTER(f64), C.POINTER(f64), pI]),
        "cvlbm2d_batch_launch_grid": (i32, [pI, C.POINTER(i32), C.POINTER(i32)]),
        "cvlbm2d_batch_destroy": (None, [pI]),
        "cvlbm_gemm_bf16": (i32, [pI, pI, pI, i32, i32, i32, i32, i32, i32, i32, pI, pI, i64,
                                  pI]),
        "cvlbm_gemm_bf16_workspace": (i64, [i32, i32, i32]),
        "cvlbm_fno_pointwise_fwd": (i32, [i32, i32, i32, i32, pI, pI, pI, pI, i32, pI, pI, pI]),
        "cvlbm_fno_gelu_bwd": (i32, [i64, pI, pI, pI, pI]),
        "cvlbm_fno_pointwise_bwd": (i32, [i32, i32, i32, i32, pI, pI, pI, pI, i32, pI, pI, pI,
                                          pI]),
        "cvlbm_fno_pointwise_scratch": (i64, [i32, i32, i32, i32]),
        "cvlbm_fno_spec_mix_fwd": (i32, [i32, i32, i32, pI, pI, pI, pI]),
        "cvlbm_fno_spec_mix_bwd": (i32, [i32, i32, i32, pI, pI, pI, pI, pI, pI]),
        "cvlbm_fno_to_bf16": (i32, [i64, pI, pI, pI]),
        "cvlbm_fno_mse": (i32, [i32, i32, i32, pI, pI, pI, pI, C.c_float, pI, pI, i32, pI]),
        "cvlbm_fno_adam": (i32, [i64, pI, pI, pI, pI, C.c_float, C.c_float, C.c_float,
                                 C.c_float, pI]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    # a library built from another header would read these structs with
    # another layout: refuse it before any call can pass one
    mirrors = (Problem2D, Fields2D, Problem3D, Fields3D, StencilInput3D)
    for which, cls in enumerate(mirrors):
        have = int(lib.cvlbm_struct_size(which))
        if have != C.sizeof(cls):
            raise RuntimeError(
                f"{path} was built for another ABI: sizeof({cls.__name__}) is {have} there and "
                f"{C.sizeof(cls)} in this binding; rebuild it (curved_lbm._build.build())")
    _lib = lib
    return lib


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = load().cvlbm_last_error()
        text = msg.decode() if msg else ""
        raise RuntimeError(f"{what} failed with code {rc}: {text}")


def torch_device(device: str | None):
    """Resolve a device string to a CUDA torch.device; CPU is rejected."""
    import torch

    name = device or os.environ.get("WARP_DEVICE") or "cuda:0"
    if not str(name).startswith("cuda"):
        raise ValueError(
            f"device {name!r} is not supported: this implementation runs only on CUDA devices")
    if not torch.cuda.is_available():
        raise RuntimeError("a CUDA device is required (no CPU fallback)")
    return torch.device(name)


def stream_ptr(device) -> int:
    import torch

    return int(torch.cuda.current_stream(device).cuda_stream)


def ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


class KernelTimer:
    """CUDA-event pairs around the dominant kernel of every step (see cvlbm.h)."""

    def __init__(self, capacity: int, kernel: str = "node") -> None:
        """kernel: "node" (the bulk node kernel) or "links" (the 2-D cut-link kernel)."""
        self.lib = load()
        self.handle = C.c_void_p()
        self._attach = (self.lib.cvlbm_timer_attach_links if kernel == "links"
                        else self.lib.cvlbm_timer_attach)
        check(self.lib.cvlbm_timer_create(int(capacity), C.byref(self.handle)), "cvlbm_timer_create")

    def attach(self) -> None:
        check(self._attach(self.handle), "cvlbm_timer_attach")

    def detach(self) -> None:
        check(self._attach(None), "cvlbm_timer_attach")

    def reset(self) -> None:
        check(self.lib.cvlbm_timer_reset(self.handle), "cvlbm_timer_reset")

    def elapsed(self) -> tuple[float, int]:
        ms, n = C.c_double(0.0), C.c_int32(0)
        check(self.lib.cvlbm_timer_elapsed(self.handle, C.byref(ms), C.byref(n)), "cvlbm_timer_elapsed")
        return float(ms.value), int(n.value)

    def __del__(self) -> None:
        try:
            self.lib.cvlbm_timer_destroy(self.handle)
        except Exception:
            pass


def launch_count() -> int:
    return int(load().cvlbm_launch_count())


def field_summary(lib, dim: int, n: int, U, u, active, device) -> dict:
    """Device reductions of summary(): max |u|, max |v|, min J, max J, finite."""
    import torch

    work = torch.empty(int(lib.cvlbm_field_summary_work_bytes()) // 8 + 1, dtype=torch.float64,
                       device=device)
    out = (f64 * 6)()
    check(lib.cvlbm_field_summary(int(dim), int(n), ptr(U), ptr(u), ptr(active), ptr(work), out,
                                  stream_ptr(device)), "cvlbm_field_summary")
    return {"max_abs_u": out[0], "max_abs_v": out[1], "min_J": out[2], "max_J": out[3],
            "finite": bool(out[4] != 0.0), "count": int(out[5])}

