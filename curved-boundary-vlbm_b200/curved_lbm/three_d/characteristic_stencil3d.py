"""Fixed geometry weights of the D3Q6 local characteristic closure, on the GPU.

Drop-in for the reference module of the same name (``build_characteristic_weights``,
three_d/characteristic_stencil3d.py:18-171): same arguments, same output
dictionary and layout, same ``ValueError``s.  The work is one launch of the
``k3_char_stencil`` kernel (``cvlbm3d_build_char_stencil`` in libcvlbm.so),
one warp per cut link: candidate ranking over the 7^3 cube, the weighted
quadratic least-squares gradient weights (normal matrix, condition check,
LU solve) and the trilinear probe weights.  The host only uploads the link
tables and reads the result back.

The gradient weights agree with the reference's LAPACK solve to round-off
(about 1e-14 of each link's largest weight); the sample choice, the probe
weights and the probe modes agree exactly.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _native

MAX_GRADIENT_SAMPLES = 48
MAX_PROBE_SAMPLES = 16
MAX_CHARACTERISTIC_SAMPLES = MAX_GRADIENT_SAMPLES + MAX_PROBE_SAMPLES
STENCIL_RADIUS = 3


def build_characteristic_weights(geometry, tables, *, batch_size=1024, link_mask=None,
                                 device=None):
    """Gradient and value-predictor weights of every (selected) cut link.

    `tables` must hold ``active_id`` (dense map lattice node -> active id,
    -1 when inactive).  `link_mask` selects the links to build (the others
    get index -1 and weight 0); `batch_size` is accepted for the reference's
    signature and has no effect (all links are built by one launch).
    """
    import torch

    nlinks = int(geometry.n_links)
    mask = None
    if link_mask is not None:
        mask = np.asarray(link_mask, dtype=bool)
        if mask.shape != (nlinks,):
            raise ValueError("link_mask must select one entry per cut link")
    spacing = np.array((geometry.dx, geometry.dy, geometry.dz), dtype=np.float64)
    if not np.allclose(spacing, spacing[0], rtol=1e-12, atol=0.0):
        raise ValueError("local_f requires an isotropic reference lattice")
    dev = _native.torch_device(device)
    lib = _native.load()

    def i32(a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)

    def f64(a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)

    act = np.asarray(geometry.active)
    keep = {"active_id": i32(tables["active_id"]).reshape(-1)}
    for k in ("i", "j", "k", "q"):
        keep["link_" + k] = i32(getattr(geometry, "link_" + k))
    for k in ("eta", "xb", "yb", "zb", "nx", "ny", "nz"):
        keep["link_" + k] = f64(getattr(geometry, "link_" + k))
    if mask is not None:
        keep["link_mask"] = torch.as_tensor(mask.astype(np.uint8), device=dev)
    idx = torch.empty((MAX_CHARACTERISTIC_SAMPLES, max(nlinks, 1)), dtype=torch.int32, device=dev)
    w = torch.empty((4, MAX_CHARACTERISTIC_SAMPLES, max(nlinks, 1)), dtype=torch.float64,
                    device=dev)
    modes = torch.zeros(max(nlinks, 1), dtype=torch.int32, device=dev)
    status = torch.zeros(max(nlinks, 1), dtype=torch.int32, device=dev)
    inp = _native.StencilInput3D()
    inp.nx, inp.ny, inp.nz = (int(v) for v in act.shape)
    inp.n_links, inp.dx = nlinks, float(spacing[0])
    for name, t in keep.items():
        setattr(inp, name, _native.ptr(t))
    _native.check(lib.cvlbm3d_build_char_stencil(C.byref(inp), _native.ptr(idx), _native.ptr(w),
                                                 _native.ptr(modes), _native.ptr(status),
                                                 _native.stream_ptr(dev)),
                  "cvlbm3d_build_char_stencil")
    st = status.cpu().numpy()[:nlinks]
    if np.any(st == 1):
        bad = np.flatnonzero(st == 1)[:8]
        raise ValueError(
            f"local_f needs a full-rank quadratic stencil within three cells; cut links {bad.tolist()}")
    if np.any(st == 2):
        raise ValueError(f"invalid local_f gradient weights near link {int(np.flatnonzero(st == 2)[0])}")
    out = {
        "indices": np.ascontiguousarray(idx.cpu().numpy()[:, :nlinks]),
        "weights": np.ascontiguousarray(w.cpu().numpy()[:, :, :nlinks]),
        "probe_modes": modes.cpu().numpy()[:nlinks].copy(),
        "radius": STENCIL_RADIUS,
        "gradient_samples": MAX_GRADIENT_SAMPLES,
        "max_samples": MAX_CHARACTERISTIC_SAMPLES,
    }
    if mask is not None:
        out["link_mask"] = mask
    return out
