"""Two-dimensional curved-boundary D2Q4x6 hyperelastic solver (drop-in).

Same module path, names, constructor arguments, methods and errors as the
reference's ``curved_lbm.two_d.curved_boundary_warp`` (curved_lbm 1.0.0);
the time step runs in hand-written sm_100a CUDA kernels (``libcvlbm.so``)
on PyTorch CUDA buffers instead of Warp kernels.  Reference line numbers are
cited per method.

Supported boundary reconstructions: ``bfl``, ``lsq_bfl``/``normal_probe_bfl``,
``compat_bfl``, ``local_char2``, ``local_f`` and ``local_f_bfl``, with the BGK
or the ``mrt_ghost`` collision and the optional kinetic ghost filter.  The
other diagnostic closures of the reference (qbfl, regularized_*, *_nee,
poly_ibb, lowq_reg_bfl) are not implemented and raise ``NotImplementedError``
at construction.
"""

from __future__ import annotations

import json
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Literal

import numpy as np

from .. import _native, _stamp
from .geometry import (
    BOUNDARY_ID_INNER,
    BOUNDARY_ID_OUTER,
    MAX_BOUNDARY_IDS,
    MAX_LSQ_STENCIL,
    CircleDomain,
    CurvedBoundaryGeometry,
    build_boundary_lsq_weights as _build_boundary_lsq_weights,
)
from .vector_nonlinear_elastic_warp import (
    BC_DIRICHLET,
    BC_NEUMANN,
    FQ,
    MATERIAL_NEO_HOOKE,
    NCOMP,
    PI,
    Q,
    SOURCE_CONSTANT,
    SOURCE_DAMPING,
    SOURCE_NONE,
    VALUE_AFFINE_VELOCITY,
    VALUE_CONSTANT,
    VALUE_ZERO,
    WarpHyperelasticMaterial,
    _CX,
    _CY,
    _equilibrium_np,
    _first_piola_np,
    _second_order_populations_masked_np,
    _second_order_populations_np,
    _source_np,
    default_device,
    source_id,
    source_name,
)

CURVED_VALUE_ZERO = VALUE_ZERO
CURVED_VALUE_CONSTANT_VECTOR = VALUE_CONSTANT
CURVED_VALUE_AFFINE_VELOCITY = VALUE_AFFINE_VELOCITY
CURVED_VALUE_PIOLA_NORMAL = 101
CURVED_VALUE_RADIAL_TRACTION = 102
CURVED_VALUE_RADIAL_TRACTION_SINE2_HOLD = 103
CURVED_VALUE_RADIAL_TRACTION_SINE2_PULSE = 104
# Not in the reference: radial traction amp*min(t/ramp_time, 1)*n,
# params (amp, ramp_time).  Used by the linear-ramp traction workloads.
CURVED_VALUE_RADIAL_TRACTION_LINEAR_HOLD = 105

BOUNDARY_RECON_BFL = 0
BOUNDARY_RECON_QBFL = 1
BOUNDARY_RECON_LSQ_BFL = 2
BOUNDARY_RECON_REG_BFL = 3
BOUNDARY_RECON_RNEE = 4
BOUNDARY_RECON_PAIR_NEE = 5
BOUNDARY_RECON_SAME_NEE = 6
BOUNDARY_RECON_POLY = 7
BOUNDARY_RECON_LOWQ_REG_BFL = 8
BOUNDARY_RECON_COMPAT_BFL = 9
BOUNDARY_RECON_COMPAT_NEE = 10
BOUNDARY_RECON_LOCAL_CHAR2 = 11
BOUNDARY_RECON_LOCAL_F = 12
BOUNDARY_RECON_LOCAL_F_BFL = 13

SUPPORTED_RECONSTRUCTIONS = (
    BOUNDARY_RECON_BFL,
    BOUNDARY_RECON_LSQ_BFL,
    BOUNDARY_RECON_COMPAT_BFL,
    BOUNDARY_RECON_LOCAL_CHAR2,
    BOUNDARY_RECON_LOCAL_F,
    BOUNDARY_RECON_LOCAL_F_BFL,
)

NORMAL_JACOBIAN_FINITE_DIFFERENCE = 0
NORMAL_JACOBIAN_ACOUSTIC = 1
NORMAL_SOLVER_ENERGY = 2

_RECON_NAMES = {
    "bfl": 0, "qbfl": 1, "lsq_bfl": 2, "normal_probe_bfl": 2, "regularized_bfl": 3,
    "regularized_nee": 4, "pair_nee": 5, "same_nee": 6, "poly_ibb": 7, "lowq_reg_bfl": 8,
    "compat_bfl": 9, "compat_nee": 10, "local_char2": 11, "char2": 11, "characteristic2": 11,
    "second_order": 11, "strict2": 11, "local_f": 12, "fully_local": 12, "local_f_bfl": 13,
    "single_history": 13,
}
_RECON_CANON = {0: "bfl", 1: "qbfl", 2: "lsq_bfl", 3: "regularized_bfl", 4: "regularized_nee",
                5: "pair_nee", 6: "same_nee", 7: "poly_ibb", 8: "lowq_reg_bfl", 9: "compat_bfl",
                10: "compat_nee", 11: "local_char2", 12: "local_f", 13: "local_f_bfl"}


def neumann_solver_name(name: str | None, material: WarpHyperelasticMaterial) -> str:
    """Reference :99-114; honours XLB_NEUMANN_SOLVER."""
    value = os.environ.get("XLB_NEUMANN_SOLVER", "newton") if name is None else str(name)
    key = value.strip().lower()
    if key not in ("newton", "energy"):
        raise ValueError(f"unsupported Neumann solver: {value!r}")
    if key == "energy" and (material.id != MATERIAL_NEO_HOOKE or not np.isfinite(material.mu)
                            or not np.isfinite(material.lam) or material.mu <= 0.0
                            or material.lam < 0.0):
        raise ValueError(
            "energy Neumann solver requires quadratic-volumetric neo_hooke, mu > 0, lambda >= 0")
    return key


def normal_jacobian_id(name: str | None = None) -> int:
    """Reference :117-124; honours XLB_NORMAL_JACOBIAN."""
    value = os.environ.get("XLB_NORMAL_JACOBIAN", "acoustic") if name is None else str(name)
    key = value.strip().lower().replace("-", "_")
    if key in ("finite_difference", "finite", "fd"):
        return NORMAL_JACOBIAN_FINITE_DIFFERENCE
    if key in ("acoustic", "acoustic_tensor", "analytic", "analytical"):
        return NORMAL_JACOBIAN_ACOUSTIC
    raise ValueError(f"unsupported normal Jacobian mode: {value!r}")


def normal_jacobian_name(mode: int) -> str:
    return {0: "finite_difference", 1: "acoustic"}.get(int(mode), f"unknown({mode})")


def boundary_reconstruction_id(name: str | int) -> int:
    if isinstance(name, int):
        return int(name)
    key = str(name).strip().lower()
    if key not in _RECON_NAMES:
        raise ValueError(f"unsupported boundary_reconstruction: {name}")
    return _RECON_NAMES[key]


def boundary_reconstruction_name(rid: int) -> str:
    return _RECON_CANON.get(int(rid), f"unknown_{rid}")


def boundary_reconstruction_stencil_radius(rid: int) -> int:
    """Maximum grid-cell radius read by one reconstruction (reference :210-222)."""
    if rid in (2, 9, 10, 11, 12):
        return 3
    if rid in (1, 7):
        return 2
    return 1


BoundaryKind = Literal["dirichlet", "neumann"]


@dataclass(frozen=True)
class CurvedBoundarySpec:
    """Physical boundary data of all cut links (reference :232-305)."""

    kind: BoundaryKind = "dirichlet"
    value_mode: int = CURVED_VALUE_ZERO
    params: tuple[float, ...] = ()
    id_kinds: dict | None = None
    id_value_modes: dict | None = None
    id_params: dict | None = None
    label: str = ""

    @property
    def kind_id(self) -> int:
        if self.kind == "dirichlet":
            return BC_DIRICHLET
        if self.kind == "neumann":
            return BC_NEUMANN
        raise ValueError(f"unsupported curved boundary kind: {self.kind}")

    @property
    def params8(self) -> np.ndarray:
        out = np.zeros(8, dtype=np.float64)
        for i, v in enumerate(self.params[:8]):
            out[i] = float(v)
        return out

    def tables(self, max_ids: int = MAX_BOUNDARY_IDS):
        kind = np.full(max_ids, self.kind_id, dtype=np.int32)
        mode = np.full(max_ids, int(self.value_mode), dtype=np.int32)
        params = np.tile(self.params8[None, :], (max_ids, 1))
        for bid, v in (self.id_kinds or {}).items():
            if 0 <= int(bid) < max_ids:
                if v == "dirichlet":
                    kind[int(bid)] = BC_DIRICHLET
                elif v == "neumann":
                    kind[int(bid)] = BC_NEUMANN
                else:
                    raise ValueError(f"unsupported boundary kind for id {bid}: {v}")
        for bid, v in (self.id_value_modes or {}).items():
            if 0 <= int(bid) < max_ids:
                mode[int(bid)] = int(v)
        for bid, vals in (self.id_params or {}).items():
            if 0 <= int(bid) < max_ids:
                params[int(bid), :] = 0.0
                for i, v in enumerate(tuple(vals)[:8]):
                    params[int(bid), i] = float(v)
        return kind, mode, np.ascontiguousarray(params)


TILE_J = 32
DEFAULT_TILE_VARIANT = 0


def _tile_list(active: np.ndarray, tile_i: int):
    """Ids (ti * tiles_j + tj) of the tile_i x 32 node tiles holding an active node."""
    nx, ny = active.shape
    ti, tj = -(-nx // tile_i), -(-ny // TILE_J)
    pad = np.zeros((ti * tile_i, tj * TILE_J), dtype=bool)
    pad[:nx, :ny] = active
    occupied = pad.reshape(ti, tile_i, tj, TILE_J).any(axis=(1, 3))
    return np.flatnonzero(occupied.reshape(-1)).astype(np.int32), tj


def _split_tiles(tiles: np.ndarray, tiles_j: int, tile_i: int, link_node: np.ndarray,
                 need: np.ndarray, halo: int = 3):
    """Tiles reordered inner first, and the inner count.

    A tile is inner when no cut-link node lies in the tile or its `halo`-node
    margin (the region the fused kernel reads populations from) and no node a
    link reads (`need`) lies in the tile.  Inner tiles of one step neither
    read what the link kernel of the previous step writes nor write what it
    reads, so the two can run at the same time.
    """
    nx, ny = link_node.shape

    def box_sums(mask):
        c = np.zeros((nx + 1, ny + 1), dtype=np.int64)
        c[1:, 1:] = mask.astype(np.int64).cumsum(0).cumsum(1)
        return c

    def count(c, i0, i1, j0, j1):
        i0, j0 = np.clip(i0, 0, nx), np.clip(j0, 0, ny)
        i1, j1 = np.clip(i1, 0, nx), np.clip(j1, 0, ny)
        return c[i1, j1] - c[i0, j1] - c[i1, j0] + c[i0, j0]

    cl, cn = box_sums(link_node), box_sums(need)
    t = np.asarray(tiles, dtype=np.int64)
    i0, j0 = (t // tiles_j) * tile_i, (t % tiles_j) * TILE_J
    inner = ((count(cl, i0 - halo, i0 + tile_i + halo, j0 - halo, j0 + TILE_J + halo) == 0)
             & (count(cn, i0, i0 + tile_i, j0, j0 + TILE_J) == 0))
    order = np.concatenate([t[inner], t[~inner]]).astype(np.int32)
    return order, int(inner.sum())


def _fused_tables(geometry, lsq_i, lsq_j, lsq_valid):
    """Tables of the fused step: link-stencil nodes and link partners.

    (The tile list depends on the fused-kernel variant; see `_tile_list`.)

    * need: nodes whose post-step U and u some cut link reads (the cut node,
      two upstream nodes along the link, and the probe/LSQ stencil);
    * partner: for link (x, q_out), the link (x, q_in) at the same node, whose
      stored outgoing population is this link's f_post[q_in](x) when the
      upstream neighbour is not active; -1 if that neighbour is active.
    """
    nx, ny = geometry.nx, geometry.ny
    act = geometry.active.astype(bool)
    need = np.zeros((nx, ny), dtype=np.uint8)
    li, lj, lq = geometry.link_i, geometry.link_j, geometry.link_q
    cx, cy = _CX[lq], _CY[lq]
    for k in range(3):
        ii, jj = li - k * cx, lj - k * cy
        ok = (ii >= 0) & (ii < nx) & (jj >= 0) & (jj < ny)
        need[ii[ok], jj[ok]] = 1
    if lsq_i is not None and len(lsq_i):
        sel = (lsq_i >= 0) & (lsq_j >= 0)
        need[lsq_i[sel], lsq_j[sel]] = 1
    key = {(int(a), int(b), int(q)): e for e, (a, b, q) in enumerate(zip(li, lj, lq))}
    partner = np.full(li.size, -1, dtype=np.int32)
    for e, (a, b, q) in enumerate(zip(li, lj, lq)):
        qi = (int(q) + 2) % 4
        ui, uj = int(a) - int(_CX[q]), int(b) - int(_CY[q])
        if not (0 <= ui < nx and 0 <= uj < ny and act[ui, uj]):
            partner[e] = key.get((int(a), int(b), qi), -1)
            if partner[e] < 0:
                return None  # link tables without the opposite link: no fused step
    return np.ascontiguousarray(need.reshape(-1)), partner


def _node_link_csr(link_node: np.ndarray, n_nodes: int):
    """CSR of link ids per node, ascending link id within a node."""
    order = np.argsort(link_node, kind="stable").astype(np.int32)
    counts = np.bincount(link_node, minlength=n_nodes) if link_node.size else np.zeros(n_nodes, np.int64)
    start = np.zeros(n_nodes + 1, dtype=np.int32)
    np.cumsum(counts, out=start[1:])
    return start, np.ascontiguousarray(order)


class WarpCurvedBoundaryLBM2D:
    """Vectorial hyperelastic LBM on an implicit 2-D domain, sm_100a kernels.

    Reference class: ``WarpCurvedBoundaryLBM2D`` (:3618-4472).  Buffers are
    torch CUDA tensors with the reference's array shapes without the trailing
    unit axis: ``f0, f1, fpost`` (24, nx, ny), ``U`` (6, nx, ny), ``u``,
    ``u_star`` (2, nx, ny), ``P, sigma`` (4, nx, ny).
    """

    def __init__(self, geometry: CurvedBoundaryGeometry, *, material: WarpHyperelasticMaterial,
                 boundary: CurvedBoundarySpec, lattice_speed: float = 5.0,
                 collision_omega: float = 2.0, collision_model: str = "bgk",
                 ghost_omega: float | None = None, kinetic_filter_strength: float = 0.0,
                 boundary_reconstruction: str = "bfl", device: str | None = None,
                 check_linearized_cfl: bool = True, jacobian_floor: float = 1.0e-12,
                 source_mode: str = "none", source_vector: tuple = (0.0,) * 6,
                 damping_gamma: float = 0.0, compatibility_projection_interval: int = 0,
                 compatibility_projection_iterations: int = 160,
                 compatibility_projection_relax: float = 0.85,
                 compatibility_projection_weight: float = 20.0,
                 compatibility_projection_repair_F: bool = False,
                 compatibility_projection_repair_F_band_width: int = -1,
                 compatibility_projection_repair_F_blend: float = 1.0,
                 compatibility_projection_boundary_id: int = BOUNDARY_ID_INNER,
                 local_compatibility_interval: int = 0, local_compatibility_blend: float = 0.05,
                 local_compatibility_interior_only: bool = True,
                 local_displacement_interval: int = 0, local_displacement_sweeps: int = 1,
                 local_displacement_relax: float = 0.85,
                 local_displacement_boundary_weight: float = 20.0,
                 local_displacement_boundary_id: int = BOUNDARY_ID_INNER,
                 normal_jacobian: str | None = None, neumann_solver: str | None = None) -> None:
        import torch

        self.geometry = geometry
        self.nx, self.ny = int(geometry.nx), int(geometry.ny)
        self.length_x, self.length_y = float(geometry.length_x), float(geometry.length_y)
        self.dx, self.dy = geometry.dx, geometry.dy
        self.material = material
        self.boundary = boundary
        self.lattice_speed = float(lattice_speed)
        self.collision_omega = float(collision_omega)
        if not (0.0 < self.collision_omega <= 2.0):
            raise ValueError("collision_omega must be in (0,2]")
        if collision_model not in ("bgk", "mrt_ghost"):
            raise ValueError("collision_model must be 'bgk' or 'mrt_ghost'")
        self.collision_model = str(collision_model)
        self.ghost_omega = float(self.collision_omega if ghost_omega is None else ghost_omega)
        if not (0.0 < self.ghost_omega <= 2.0):
            raise ValueError("ghost_omega must be in (0,2]")
        self.kinetic_filter_strength = float(kinetic_filter_strength)
        if not (0.0 <= self.kinetic_filter_strength <= 1.0):
            raise ValueError("kinetic_filter_strength must be in [0,1]")
        self.boundary_reconstruction = boundary_reconstruction_id(str(boundary_reconstruction))
        self.boundary_reconstruction_name = boundary_reconstruction_name(self.boundary_reconstruction)
        self.boundary_stencil_radius = boundary_reconstruction_stencil_radius(
            self.boundary_reconstruction)
        self.normal_jacobian = normal_jacobian_id(normal_jacobian)
        self.normal_jacobian_name = normal_jacobian_name(self.normal_jacobian)
        self.neumann_solver_name = neumann_solver_name(neumann_solver, material)
        self._normal_solver_mode = (NORMAL_SOLVER_ENERGY if self.neumann_solver_name == "energy"
                                    else self.normal_jacobian)
        if check_linearized_cfl and material.linearized_stability_ratio(self.lattice_speed) >= 1.0:
            raise ValueError("linearized D2Q4 stability ratio must be below one")
        self.dt = self.dx / self.lattice_speed
        self.time = 0.0
        self.steps = 0
        self.jacobian_floor = float(jacobian_floor)
        self.shape = (self.nx, self.ny, 1)
        self.source_mode = source_id(source_mode)
        self._source_name_func = source_name
        self.source_params = np.zeros(NCOMP, dtype=np.float64)
        if self.source_mode == SOURCE_CONSTANT:
            for i, v in enumerate(tuple(source_vector)[:NCOMP]):
                self.source_params[i] = float(v)
        elif self.source_mode == SOURCE_DAMPING:
            if damping_gamma < 0.0:
                raise ValueError("damping_gamma must be non-negative")
            self.source_params[0] = float(damping_gamma)
        if int(compatibility_projection_interval) != 0:
            raise ValueError("the fully-local solver forbids compatibility_projection_interval != 0")
        self.compatibility_projection_interval = 0
        self.compatibility_projection_iterations = int(max(1, compatibility_projection_iterations))
        self.compatibility_projection_relax = float(compatibility_projection_relax)
        self.compatibility_projection_weight = float(compatibility_projection_weight)
        self.compatibility_projection_repair_F = False
        self.compatibility_projection_repair_F_band_width = int(
            compatibility_projection_repair_F_band_width)
        self.compatibility_projection_repair_F_blend = float(compatibility_projection_repair_F_blend)
        self.compatibility_projection_boundary_id = int(compatibility_projection_boundary_id)
        self._compatibility_projector = None
        self.local_compatibility_interval = int(max(0, local_compatibility_interval))
        self.local_compatibility_blend = float(local_compatibility_blend)
        self.local_compatibility_interior_only = bool(local_compatibility_interior_only)
        if not (0.0 <= self.local_compatibility_blend <= 1.0):
            raise ValueError("local_compatibility_blend must be in [0,1]")
        self.local_displacement_interval = int(max(0, local_displacement_interval))
        self.local_displacement_sweeps = int(local_displacement_sweeps)
        self.local_displacement_relax = float(local_displacement_relax)
        self.local_displacement_boundary_weight = float(local_displacement_boundary_weight)
        self.local_displacement_boundary_id = int(local_displacement_boundary_id)
        if not (0.0 <= self.local_displacement_relax <= 1.0):
            raise ValueError("local_displacement_relax must be in [0,1]")
        if not (1 <= self.local_displacement_sweeps <= 8):
            raise ValueError(
                "local_displacement_sweeps must be in [1,8] to keep a bounded local dependency radius")
        if self.local_displacement_boundary_weight < 0.0:
            raise ValueError("local_displacement_boundary_weight must be non-negative")
        if self.boundary_reconstruction not in SUPPORTED_RECONSTRUCTIONS:
            raise NotImplementedError(
                f"boundary_reconstruction={self.boundary_reconstruction_name!r} is not implemented")

        self.device = str(device or default_device())
        self._tdev = _native.torch_device(self.device)
        self._lib = _native.load()
        dev, f64, i32 = self._tdev, torch.float64, torch.int32

        def dev_i(a):
            return torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)

        def dev_f(a):
            return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)

        x = (np.arange(self.nx, dtype=np.float64) + 0.5) * self.dx
        y = (np.arange(self.ny, dtype=np.float64) + 0.5) * self.dy
        self.x, self.y = np.meshgrid(x, y, indexing="ij")
        self.active_np = np.ascontiguousarray(geometry.active.astype(np.int32))
        nl = int(geometry.n_links)
        if geometry.lsq_i is None or geometry.lsq_j is None or geometry.lsq_wb is None \
                or geometry.lsq_valid is None:
            lsq_i = np.full((nl, MAX_LSQ_STENCIL), -1, np.int32)
            lsq_j = np.full((nl, MAX_LSQ_STENCIL), -1, np.int32)
            zeros = np.zeros((nl, MAX_LSQ_STENCIL))
            lsq_wb, lsq_wt, lsq_wx, lsq_wy = zeros, zeros, zeros, zeros
            lsq_valid = np.zeros(nl, np.int32)
        else:
            lsq_i, lsq_j, lsq_wb = geometry.lsq_i, geometry.lsq_j, geometry.lsq_wb
            zl = np.zeros_like(lsq_wb)
            lsq_wt = geometry.lsq_wt if geometry.lsq_wt is not None else zl
            lsq_wx = geometry.lsq_wx if geometry.lsq_wx is not None else zl
            lsq_wy = geometry.lsq_wy if geometry.lsq_wy is not None else zl
            lsq_valid = geometry.lsq_valid
        self.lsq_wb_np = np.asarray(lsq_wb, dtype=np.float64)
        self.lsq_wt_np = np.asarray(lsq_wt, dtype=np.float64)
        self.lsq_wx_np = np.asarray(lsq_wx, dtype=np.float64)
        self.lsq_wy_np = np.asarray(lsq_wy, dtype=np.float64)
        self.lsq_valid_np = np.asarray(lsq_valid, dtype=np.int32)
        self.boundary_params = boundary.params8
        kind, mode, params = boundary.tables(MAX_BOUNDARY_IDS)
        self.boundary_kind_by_id_np, self.boundary_mode_by_id_np = kind, mode
        self.boundary_params_by_id_np = params

        link_node = (geometry.link_i.astype(np.int64) * self.ny + geometry.link_j).astype(np.int64)
        start, order = _node_link_csr(link_node, self.nx * self.ny)
        t = {}
        t["active"] = dev_i(self.active_np.reshape(-1))
        for name in ("link_i", "link_j", "link_q"):
            t[name] = dev_i(getattr(geometry, name))
        t["link_bid"] = dev_i(geometry.link_boundary_id)
        for name in ("link_eta", "link_xb", "link_yb", "link_nx", "link_ny"):
            t[name] = dev_f(getattr(geometry, name))
        t["lsq_i"], t["lsq_j"] = dev_i(lsq_i), dev_i(lsq_j)
        t["lsq_wb"], t["lsq_wt"] = dev_f(lsq_wb), dev_f(lsq_wt)
        t["lsq_wx"], t["lsq_wy"] = dev_f(lsq_wx), dev_f(lsq_wy)
        t["lsq_valid"] = dev_i(lsq_valid)
        t["node_link_start"], t["node_link_list"] = dev_i(start), dev_i(order)
        t["bc_kind"], t["bc_mode"], t["bc_params"] = dev_i(kind), dev_i(mode), dev_f(params)
        fused = _fused_tables(geometry, np.asarray(lsq_i), np.asarray(lsq_j), lsq_valid)
        self._need_np = None
        if fused is not None:
            need, partner = fused
            self._need_np = need
            t["need_fields"] = torch.as_tensor(need, device=dev)
            t["link_partner"] = dev_i(partner)
        self._tile_lists: dict = {}
        self._fused_possible = fused is not None
        self.tile_variant = DEFAULT_TILE_VARIANT
        li_np, lj_np = np.asarray(lsq_i), np.asarray(lsq_j)
        t["lsq_node"] = dev_i(np.where((li_np >= 0) & (lj_np >= 0), li_np * self.ny + lj_np, -1))
        # traction (Neumann) links first, then by node: a warp's links share branches
        link_kind = kind[np.clip(geometry.link_boundary_id, 0, MAX_BOUNDARY_IDS - 1)]
        order = np.lexsort((np.arange(nl), link_kind != BC_NEUMANN))
        t["link_order"] = dev_i(order)
        # the link kernel's first loads, one row per processing slot
        rows = np.zeros(nl, dtype=_native.link_row2_dtype())
        li_o, lj_o, lq_o = (np.asarray(getattr(geometry, k))[order].astype(np.int64)
                            for k in ("link_i", "link_j", "link_q"))
        rows["ell"], rows["i"], rows["j"], rows["q"] = order, li_o, lj_o, lq_o
        rows["node"] = li_o * self.ny + lj_o
        ui, uj = li_o - _CX[lq_o], lj_o - _CY[lq_o]
        inb = (ui >= 0) & (ui < self.nx) & (uj >= 0) & (uj < self.ny)
        up_act = np.zeros(nl, dtype=bool)
        up_act[inb] = self.active_np[ui[inb], uj[inb]] != 0
        rows["upstream"] = np.where(up_act, ui * self.ny + uj, -1)
        bid = np.asarray(geometry.link_boundary_id)[order]
        rows["bid"] = np.where((bid >= 0) & (bid < MAX_BOUNDARY_IDS), bid, 0)
        rows["lsq_valid"] = np.asarray(lsq_valid)[order]
        for k in ("eta", "xb", "yb", "nx", "ny"):
            rows[k] = np.asarray(getattr(geometry, "link_" + k))[order]
        t["link_rows"] = torch.as_tensor(rows.view(np.uint8), device=dev)
        lsq_node_np = np.where((li_np >= 0) & (lj_np >= 0), li_np * self.ny + lj_np, -1)
        t["lsq_node_slot"] = dev_i(np.asarray(lsq_node_np)[order])
        for k, w in (("wb", lsq_wb), ("wt", lsq_wt), ("wx", lsq_wx), ("wy", lsq_wy)):
            t[f"lsq_{k}_slot"] = dev_f(np.asarray(w)[order])
        self.link_scratch = torch.zeros(max(6 * nl, 1), dtype=f64, device=dev)
        self.link_traction_x = torch.zeros(nl, dtype=f64, device=dev)
        self.link_traction_y = torch.zeros(nl, dtype=f64, device=dev)
        self.use_dynamic_link_traction = False
        self._tables = t

        shp = (self.nx, self.ny)
        self.f0 = torch.zeros((FQ,) + shp, dtype=f64, device=dev)
        self.f1 = torch.zeros_like(self.f0)
        self.fpost = torch.zeros_like(self.f0)
        self.U = torch.zeros((NCOMP,) + shp, dtype=f64, device=dev)
        self.u = torch.zeros((2,) + shp, dtype=f64, device=dev)
        self.u_star = torch.zeros_like(self.u)
        self.u_local_next = torch.zeros_like(self.u)
        self.P = torch.zeros((4,) + shp, dtype=f64, device=dev)
        self.sigma = torch.zeros_like(self.P)
        self.invalid = torch.zeros(1, dtype=i32, device=dev)
        self._clock = torch.zeros(2, dtype=f64, device=dev)
        self._stress_current = True
        self._graphs: dict = {}
        self.use_graphs = True
        self._problem = self._make_problem()
        self._select_variant(self.tile_variant)
        self.initialize_identity(init_order=1)

    # -- native plumbing ---------------------------------------------------
    @property
    def overlap_links(self) -> bool:
        """Run the next step's inner tiles on a second stream while the cut-link
        kernel runs (fused step only; results are identical either way)."""
        return bool(self._problem.overlap)

    @overlap_links.setter
    def overlap_links(self, on: bool) -> None:
        self._problem.overlap = int(bool(on))

    def _select_variant(self, variant: int) -> None:
        """Point the problem at the tile list of fused-kernel variant `variant`."""
        import torch

        tile_i = int(self._lib.cvlbm2d_tile_variant(int(variant)))
        if tile_i <= 0:
            raise ValueError(f"fused-kernel variant {variant} is not compiled")
        if tile_i not in self._tile_lists:
            tiles, tj = _tile_list(self.active_np.astype(bool), tile_i)
            n_inner = 0
            if self._need_np is not None:
                link_node = np.zeros((self.nx, self.ny), dtype=bool)
                link_node[self.geometry.link_i, self.geometry.link_j] = True
                tiles, n_inner = _split_tiles(
                    tiles, tj, tile_i, link_node,
                    np.asarray(self._need_np).reshape(self.nx, self.ny).astype(bool))
            self._tile_lists[tile_i] = (torch.as_tensor(tiles, device=self._tdev), tj, n_inner)
        tiles, tj, n_inner = self._tile_lists[tile_i]
        self._tables["tiles"] = tiles
        self.tile_variant = int(variant)
        p = self._problem
        p.tile_variant, p.tile_i = int(variant), tile_i
        p.n_tiles, p.tiles_j = int(tiles.numel()), int(tj)
        p.n_tiles_inner = int(n_inner)
        p.tiles = _native.ptr(tiles) if self._fused_possible else None

    def autotune(self, steps: int = 40, variants=None) -> dict:
        """Time every compiled fused-kernel variant on this problem; keep the fastest.

        Runs on a copy of the state (populations, u*, time) that is restored
        afterwards, so the solution is unchanged.  Returns {variant: us/step}.
        """
        import torch

        if not self._fused_possible:
            return {}
        saved = (self.f0.clone(), self.f1.clone(), self.u_star.clone(), self.U.clone(),
                 self.u.clone(), self.time, self.steps)
        cand = [v for v in (variants if variants is not None else range(16))
                if int(self._lib.cvlbm2d_tile_variant(int(v))) > 0]
        times = {}
        use_graphs, self.use_graphs = self.use_graphs, False  # time launches, not captures
        for v in cand:
            self._select_variant(v)
            self.run(4)
            torch.cuda.synchronize(self._tdev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self.run(steps)
            e1.record()
            e1.synchronize()
            times[v] = e0.elapsed_time(e1) * 1e3 / steps
            self.f0.copy_(saved[0]); self.f1.copy_(saved[1]); self.u_star.copy_(saved[2])
            self.U.copy_(saved[3]); self.u.copy_(saved[4])
            self.time, self.steps = saved[5], saved[6]
        self.use_graphs = use_graphs
        best = min(times, key=times.get)
        self._select_variant(best)
        return times
    def _make_problem(self) -> _native.Problem2D:
        t = self._tables
        m = self.material
        p = _native.Problem2D()
        p.nx, p.ny, p.n_links = self.nx, self.ny, int(self.geometry.n_links)
        p.recon = int(self.boundary_reconstruction)
        p.normal_solver = int(self._normal_solver_mode)
        p.source_mode = int(self.source_mode)
        p.dx, p.dy, p.dt = self.dx, self.dy, self.dt
        p.omega, p.c = self.collision_omega, self.lattice_speed
        for i in range(6):
            p.source[i] = float(self.source_params[i])
        p.mat = _native.Material(int(m.id), 0, float(m.lam), float(m.mu), float(m.param0),
                                 float(m.param1), float(m.param2), self.jacobian_floor)
        p.disp_interval = self.local_displacement_interval
        p.disp_sweeps = self.local_displacement_sweeps
        p.disp_bid = self.local_displacement_boundary_id
        p.rep_interval = self.local_compatibility_interval
        p.interior_only = int(self.local_compatibility_interior_only)
        p.use_dynamic_traction = int(self.use_dynamic_link_traction)
        p.relax = self.local_displacement_relax
        p.weight = self.local_displacement_boundary_weight
        p.blend = self.local_compatibility_blend
        p.collision_model = 1 if self.collision_model == "mrt_ghost" else 0
        p.ghost_omega = self.ghost_omega
        p.kinetic_filter = self.kinetic_filter_strength
        for name, tensor in t.items():
            setattr(p, name, _native.ptr(tensor))
        p.traction_x = _native.ptr(self.link_traction_x)
        p.traction_y = _native.ptr(self.link_traction_y)
        p.overlap = 1
        return p

    def _set_fused(self, enabled: bool) -> None:
        """Select the fused node kernel (default) or the per-phase kernels."""
        t = self._tables.get("tiles")
        ok = enabled and t is not None and self._fused_possible
        self._problem.tiles = _native.ptr(t) if ok else None

    def _fields(self) -> _native.Fields2D:
        fl = _native.Fields2D()
        for name, tensor in (("f0", self.f0), ("f1", self.f1), ("fpost", self.fpost),
                             ("U", self.U), ("u", self.u), ("u_next", self.u_local_next),
                             ("u_star", self.u_star), ("P", self.P), ("sigma", self.sigma),
                             ("invalid", self.invalid), ("clock", self._clock),
                             ("link_scratch", self.link_scratch)):
            setattr(fl, name, _native.ptr(tensor))
        return fl

    def _stream(self) -> int:
        return _native.stream_ptr(self._tdev)

    # -- initialisation ----------------------------------------------------
    def initialize_identity(self, *, init_order: int = 1) -> None:
        U = np.zeros((NCOMP, self.nx, self.ny), dtype=np.float64)
        U[2] = 1.0
        U[5] = 1.0
        self.initialize_from_numpy(U=U, displacement=np.zeros((2, self.nx, self.ny)),
                                   init_order=init_order)

    def initialize_from_numpy(self, *, U: np.ndarray, displacement: np.ndarray | None = None,
                              init_order: int = 1, apply_initial_boundaries: bool = True,
                              initial_boundary_time: float = 0.0) -> None:
        """Initial populations, u*, in-place boundary pass (reference :3855-3954).

        The populations are formed on the device by the operations of the
        reference's host NumPy code; where that code raises or retries (a
        flux evaluation with J <= 0), it runs on the host instead."""
        import torch

        U = np.asarray(U, dtype=np.float64)
        if U.shape != (NCOMP, self.nx, self.ny):
            raise ValueError(f"U must have shape {(NCOMP, self.nx, self.ny)}")
        disp = (np.zeros((2, self.nx, self.ny)) if displacement is None
                else np.asarray(displacement, dtype=np.float64))
        if disp.shape != (2, self.nx, self.ny):
            raise ValueError(f"displacement must have shape {(2, self.nx, self.ny)}")
        if init_order not in (1, 2, 3):
            raise ValueError("init_order must be 1, 2, or 3")
        # formed in fpost (zeroed below) so that f0 is untouched if the host
        # code raises
        if self._device_initial_populations(U, init_order, self.fpost):
            self.f0.copy_(self.fpost)
        else:
            # the host code raises FloatingPointError (or retries a flux
            # tangent with a smaller step) where the device kernels flagged
            f = self._host_initial_populations(U, init_order)
            self.f0.copy_(torch.as_tensor(np.ascontiguousarray(f.reshape((FQ, self.nx, self.ny))),
                                          device=self._tdev))
        inactive = self.active_np == 0
        dm = np.array(disp, dtype=np.float64, copy=True)
        dm[:, inactive] = 0.0
        us0 = dm - 0.5 * self.dt * U[:2]
        us0[:, inactive] = 0.0
        dev = self._tdev
        self.f1.zero_()
        self.fpost.zero_()
        self.u_star.copy_(torch.as_tensor(np.ascontiguousarray(us0), device=dev))
        self.time = 0.0
        self.steps = 0
        self._graphs.clear()
        self.refresh_current()
        if apply_initial_boundaries:
            self.apply_boundary_reconstruction(float(initial_boundary_time), in_place=True)
            if self.kinetic_filter_strength > 0.0:  # reference :3947-3952
                _native.check(self._lib.cvlbm2d_kinetic_filter(self._problem, self._fields(),
                                                               self._stream()),
                              "cvlbm2d_kinetic_filter")
            self.refresh_current()

    def _host_initial_populations(self, U: np.ndarray, init_order: int) -> np.ndarray:
        """Initial populations [4, 6, nx, ny] by the reference's host NumPy
        (:3875-3890), zero at inactive nodes."""
        if init_order == 1:
            f = _equilibrium_np(U, self.material, self.lattice_speed)
            src = _source_np(U, self.source_mode, self.source_params)
            f -= (0.5 * self.dt / float(Q)) * src[None, ...]
        elif init_order == 2:
            f = _second_order_populations_np(
                U, self.material, self.lattice_speed, dx=self.dx, dy=self.dy, dt=self.dt,
                periodic_x=False, periodic_y=False, source_mode=self.source_mode,
                source_params=self.source_params)
        else:
            f = _second_order_populations_masked_np(
                U, self.active_np.astype(bool), self.material, self.lattice_speed, dx=self.dx,
                dy=self.dy, dt=self.dt, periodic_x=False, periodic_y=False,
                source_mode=self.source_mode, source_params=self.source_params)
        f[:, :, self.active_np == 0] = 0.0
        return f

    def _device_initial_populations(self, U: np.ndarray, init_order: int, out) -> bool:
        """`out` ([24, nx, ny] device tensor) from U by the library's init
        kernels (cvlbm2d_init_populations,
        the host NumPy's operations on the device); False where the host code
        has to run instead (a flux evaluation with J <= 0 or past the Gent
        chain limit, where it raises or retries with a smaller step)."""
        import torch

        dev = self._tdev
        Ud = torch.as_tensor(np.ascontiguousarray(U.reshape(NCOMP, -1)), device=dev)
        nbytes = int(self._lib.cvlbm2d_init_work_bytes(self.nx, self.ny))
        work = torch.empty(nbytes // 8 + 1, dtype=torch.float64, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        _native.check(self._lib.cvlbm2d_init_populations(
            self._problem, _native.ptr(Ud), int(init_order), _native.ptr(out),
            _native.ptr(work), _native.ptr(status), self._stream()), "cvlbm2d_init_populations")
        return int(status.item()) == 0

    # -- boundary ----------------------------------------------------------
    def enable_dynamic_link_traction(self, enabled: bool = True) -> None:
        """Neumann links read ``link_traction_x/y[ell]`` (reference :4011-4018)."""
        self.use_dynamic_link_traction = bool(enabled)
        self._problem.use_dynamic_traction = int(self.use_dynamic_link_traction)

    def apply_boundary_reconstruction(self, boundary_time: float, *, in_place: bool = False) -> None:
        """Reference :4020-4035."""
        if self.geometry.n_links == 0:
            return
        fl = self._fields()
        _native.check(self._lib.cvlbm2d_apply_boundary(self._problem, fl, float(boundary_time),
                                                       int(bool(in_place)), self._stream()),
                      "cvlbm2d_apply_boundary")
        self._stress_current = False

    def configure_compatibility_projection(self, *, interval: int = 1, iterations: int = 160,
                                           relax: float = 0.85, weight: float = 20.0,
                                           repair_F: bool = False, repair_F_band_width: int = -1,
                                           repair_F_blend: float = 1.0,
                                           boundary_id: int = BOUNDARY_ID_INNER) -> None:
        if int(interval) != 0 or bool(repair_F):
            raise ValueError("global compatibility projection is not available in the fully-local solver")

    def project_compatible_displacement(self, *, iterations=None, repair_F=None) -> None:
        raise RuntimeError("global compatibility projection is disabled by design")

    def _compatibility_projection_due(self) -> bool:
        return False

    def _local_compatibility_due(self) -> bool:
        return self.local_compatibility_interval > 0 and self.steps % self.local_compatibility_interval == 0

    def _local_displacement_due(self) -> bool:
        return self.local_displacement_interval > 0 and self.steps % self.local_displacement_interval == 0

    # -- time stepping -----------------------------------------------------
    GRAPH_MIN_STEPS = 8   # run() replays a cached CUDA graph for even counts from here on
    GRAPH_CACHE = 8       # graphs kept per solver

    def _cached_graph(self, nsteps: int):
        """The CUDA graph of `nsteps` steps for the current buffers, settings
        and kinematic phase (captured on first use), or None when run() takes
        the plain launch path (odd or short counts, graphs switched off)."""
        import ctypes

        if not self.use_graphs or nsteps < self.GRAPH_MIN_STEPS or nsteps % 2:
            return None
        phase = tuple(self.steps % iv for iv in (self.local_displacement_interval,
                                                 self.local_compatibility_interval) if iv > 0)
        key = (nsteps, phase, ctypes.string_at(ctypes.addressof(self._problem),
                                               ctypes.sizeof(self._problem)),
               bytes(self._fields()))
        g = self._graphs.get(key)
        if g is None:
            if len(self._graphs) >= self.GRAPH_CACHE:
                self._graphs.pop(next(iter(self._graphs)))
            g = self._graphs[key] = _Graph2D(self, nsteps)
        return g

    def run(self, nsteps: int) -> None:
        """Advance ``nsteps`` steps (no host sync).  Even counts of at least
        GRAPH_MIN_STEPS replay a cached CUDA graph of the same launches (same
        results); other counts make one native call."""
        nsteps = int(nsteps)
        if nsteps <= 0:
            return
        g = self._cached_graph(nsteps)
        if g is not None:
            g.launch()
            return
        fl = self._fields()
        _native.check(self._lib.cvlbm2d_run(self._problem, fl, float(self.time), int(self.steps),
                                            nsteps, 0, self._stream()), "cvlbm2d_run")
        if nsteps % 2 == 1:
            self.f0, self.f1 = self.f1, self.f0
        for _ in range(nsteps):
            self.time += self.dt
        self.steps += nsteps
        self._stress_current = False

    def step(self) -> None:
        """One time step (reference :4163-4258)."""
        self.run(1)

    def capture_graph(self, nsteps: int):
        """CUDA graph of ``nsteps`` (even) steps starting at the current phase."""
        return _Graph2D(self, int(nsteps))

    def refresh_current(self) -> None:
        """Reference :4260-4291."""
        fl = self._fields()
        _native.check(self._lib.cvlbm2d_refresh(self._problem, fl, self._stream()),
                      "cvlbm2d_refresh")
        self._stress_current = True

    def run_until(self, t_end: float, *, stop_on_invalid: bool = True,
                  check_interval: int = 0) -> None:
        """Reference :4293-4306.  Steps run in native batches between checks."""
        import torch

        remaining = 0
        tt = self.time
        while tt < float(t_end) - 0.5 * self.dt:
            tt += self.dt
            remaining += 1
        ci = int(check_interval)
        while remaining > 0:
            if stop_on_invalid and ci > 0:
                chunk = ci - (self.steps % ci)
                chunk = min(chunk, remaining)
            else:
                chunk = remaining
            self.run(chunk)
            remaining -= chunk
            if stop_on_invalid and ci > 0 and self.steps % ci == 0 and self.invalid_state():
                break
        self.refresh_current()
        torch.cuda.synchronize(self._tdev)

    # -- outputs -----------------------------------------------------------
    def invalid_state(self) -> bool:
        """Reference :4308-4314."""
        import torch

        torch.cuda.synchronize(self._tdev)
        if int(self.invalid.item()) != 0:
            return True
        U = self.numpy_field("U")
        mask = self.active_np.astype(bool)
        return not np.isfinite(U[:, mask]).all()

    def numpy_field(self, name: str) -> np.ndarray:
        """Host copy of a field, shapes as the reference's without the unit axis."""
        import torch

        if name in ("P", "sigma") and not self._stress_current:
            _native.check(self._lib.cvlbm2d_stress(self._problem, self._fields(), self._stream()),
                          "cvlbm2d_stress")
            self._stress_current = True
        field = getattr(self, name)
        torch.cuda.synchronize(self._tdev)
        return field.detach().cpu().numpy()

    def displacement(self) -> np.ndarray:
        return self.numpy_field("u")

    def system_state(self) -> np.ndarray:
        return self.numpy_field("U")

    def deformation_gradient(self) -> np.ndarray:
        U = self.system_state()
        F = np.empty((2, 2, self.nx, self.ny), dtype=np.float64)
        F[0, 0], F[0, 1], F[1, 0], F[1, 1] = U[2], U[3], U[4], U[5]
        return F

    def deformation_jacobian(self) -> np.ndarray:
        F = self.deformation_gradient()
        return F[0, 0] * F[1, 1] - F[0, 1] * F[1, 0]

    def active_mask(self) -> np.ndarray:
        return self.active_np.astype(bool)

    def summary(self) -> dict:
        """Reference :4343-4415.  The field reductions (max |u|, max |v|,
        min / max J, finite) run on the device (cvlbm_field_summary)."""
        self.refresh_current()
        red = _native.field_summary(self._lib, 2, self.nx * self.ny, self.U, self.u,
                                    self._tables["active"], self._tdev)
        anym = red["count"] > 0
        drad = self.local_displacement_sweeps if self.local_displacement_interval > 0 else 0
        crad = drad + 2 if self.local_compatibility_interval > 0 else drad
        return {
            "device": self.device, "geometry": self.geometry.label,
            "boundary_label": self.boundary.label, "boundary_kind": self.boundary.kind,
            "boundary_mode": int(self.boundary.value_mode), "model": self.material.model,
            "lambda": float(self.material.lam), "mu": float(self.material.mu), "nx": self.nx,
            "ny": self.ny, "n_active": int(red["count"]),
            "n_cut_links": self.geometry.n_links, "steps": self.steps, "time": float(self.time),
            "dx": float(self.dx), "dt": float(self.dt), "lattice_speed": float(self.lattice_speed),
            "collision_omega": float(self.collision_omega), "collision_model": self.collision_model,
            "ghost_omega": float(self.ghost_omega),
            "kinetic_filter_strength": float(self.kinetic_filter_strength),
            "boundary_reconstruction": self.boundary_reconstruction_name,
            "boundary_stencil_radius": self.boundary_stencil_radius,
            "normal_jacobian": self.normal_jacobian_name,
            "neumann_solver": self.neumann_solver_name,
            "local_compatibility_interval": self.local_compatibility_interval,
            "local_compatibility_blend": self.local_compatibility_blend,
            "local_compatibility_interior_only": self.local_compatibility_interior_only,
            "local_displacement_interval": self.local_displacement_interval,
            "local_displacement_sweeps": self.local_displacement_sweeps,
            "local_displacement_relax": self.local_displacement_relax,
            "local_displacement_boundary_weight": self.local_displacement_boundary_weight,
            "local_displacement_boundary_id": self.local_displacement_boundary_id,
            "local_kernel_stencil_radius": 2 if self.local_compatibility_interval > 0
            else (1 if drad > 0 else 0),
            "local_displacement_dependency_radius": drad,
            "local_composed_compatibility_radius": crad,
            "linearized_stability_ratio": float(
                self.material.linearized_stability_ratio(self.lattice_speed)),
            "max_abs_u": float(red["max_abs_u"]) if anym else 0.0,
            "max_abs_v": float(red["max_abs_v"]) if anym else 0.0,
            "min_J": float(red["min_J"]) if anym else 0.0,
            "max_J": float(red["max_J"]) if anym else 0.0,
            "finite": red["finite"] if anym else False,
        }

    # -- exact checkpoint / restart (no counterpart in the reference) --------
    def _checkpoint_stamp(self) -> str:
        g = self.geometry
        return _stamp.config_stamp(
            self,
            geometry_arrays=(self.active_np, g.link_i, g.link_j, g.link_q, g.link_boundary_id,
                             g.link_eta, g.link_xb, g.link_yb, g.link_nx, g.link_ny,
                             self.lsq_wb_np, self.lsq_wt_np, self.lsq_wx_np, self.lsq_wy_np,
                             self.lsq_valid_np),
            boundary_tables=(self.boundary_kind_by_id_np, self.boundary_mode_by_id_np,
                             self.boundary_params_by_id_np))

    def checkpoint(self, path: str | Path) -> None:
        """Write the complete stepping state (populations, u*, U, u, time and
        step count) so that `restore` on a solver built with the same
        geometry and settings continues bit for bit.  (`save_npz` writes the
        reference's output format, which lacks u*.)"""
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        host = {k: t.detach().cpu().numpy() for k, t in
                (("f0", self.f0), ("u_star", self.u_star), ("U", self.U), ("u", self.u))}
        np.savez(path, **host, time=np.array(self.time), steps=np.array(self.steps),
                 stamp=np.array(self._checkpoint_stamp()))

    def restore(self, path: str | Path) -> None:
        """Load a `checkpoint` written by a solver with the same geometry and
        settings (ValueError otherwise)."""
        import torch

        d = np.load(Path(path), allow_pickle=False)
        if str(d["stamp"]) != self._checkpoint_stamp():
            raise ValueError("checkpoint was written by a solver with another configuration")
        for name, dst in (("f0", self.f0), ("u_star", self.u_star), ("U", self.U), ("u", self.u)):
            src = d[name]
            if tuple(src.shape) != tuple(dst.shape):
                raise ValueError(f"checkpoint field {name} has shape {src.shape}")
            dst.copy_(torch.as_tensor(src, device=self._tdev))
        self.time = float(d["time"])
        self.steps = int(d["steps"])
        self._stress_current = False

    def save_npz(self, path: str | Path) -> None:
        """Reference :4417-4472."""
        self.refresh_current()
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        g = self.geometry
        np.savez_compressed(
            path, x=self.x, y=self.y, active=self.active_np, u=self.displacement(),
            U=self.system_state(), F=self.deformation_gradient(), P=self.numpy_field("P"),
            sigma=self.numpy_field("sigma"), f=self.numpy_field("f0"), link_i=g.link_i,
            link_j=g.link_j, link_q=g.link_q, link_boundary_id=g.link_boundary_id,
            link_eta=g.link_eta, link_xb=g.link_xb, link_yb=g.link_yb, link_nx=g.link_nx,
            link_ny=g.link_ny, lsq_valid=self.lsq_valid_np, time=np.array(self.time),
            dx=np.array(self.dx), dt=np.array(self.dt), lattice_speed=np.array(self.lattice_speed),
            collision_omega=np.array(self.collision_omega),
            collision_model=np.array(self.collision_model), ghost_omega=np.array(self.ghost_omega),
            kinetic_filter_strength=np.array(self.kinetic_filter_strength),
            boundary_reconstruction=np.array(self.boundary_reconstruction_name),
            normal_jacobian=np.array(self.normal_jacobian_name),
            neumann_solver=np.array(self.neumann_solver_name),
            local_compatibility_interval=np.array(self.local_compatibility_interval),
            local_compatibility_blend=np.array(self.local_compatibility_blend),
            local_compatibility_interior_only=np.array(self.local_compatibility_interior_only),
            local_displacement_interval=np.array(self.local_displacement_interval),
            local_displacement_sweeps=np.array(self.local_displacement_sweeps),
            local_displacement_relax=np.array(self.local_displacement_relax),
            local_displacement_boundary_weight=np.array(self.local_displacement_boundary_weight),
            local_displacement_boundary_id=np.array(self.local_displacement_boundary_id),
            boundary_kind=np.array(self.boundary.kind),
            boundary_mode=np.array(int(self.boundary.value_mode)),
            boundary_params=self.boundary_params,
            boundary_kind_by_id=self.boundary_kind_by_id_np,
            boundary_mode_by_id=self.boundary_mode_by_id_np,
            boundary_params_by_id=self.boundary_params_by_id_np, model=np.array(self.material.model),
            lam=np.array(self.material.lam), mu=np.array(self.material.mu),
            material_params=np.asarray(self.material.params, dtype=np.float64),
            metadata=np.array(json.dumps(self.summary())))


class _Graph2D:
    """Executable CUDA graph of ``nsteps`` steps of one 2-D solver.

    Replays advance the solver exactly like ``run(nsteps)``; the time comes
    from a device clock that the graph advances.  Valid while the solver's
    buffers and configuration are unchanged and the step phase modulo the
    kinematic intervals matches the capture phase.
    """

    def __init__(self, solver: WarpCurvedBoundaryLBM2D, nsteps: int) -> None:
        import ctypes

        if nsteps <= 0 or nsteps % 2:
            raise ValueError("graph step count must be a positive even number")
        self.solver = solver
        self.nsteps = nsteps
        self.step0 = solver.steps
        handle = ctypes.c_void_p()
        _native.check(solver._lib.cvlbm2d_graph_create(solver._problem, solver._fields(),
                                                       solver.steps, nsteps, ctypes.byref(handle)),
                      "cvlbm2d_graph_create")
        self.handle = handle

    def _phase_ok(self) -> bool:
        s = self.solver
        for iv in (s.local_displacement_interval, s.local_compatibility_interval):
            if iv > 0 and (s.steps - self.step0) % iv != 0:
                return False
        return True

    def launch(self) -> None:
        s = self.solver
        if not self._phase_ok():
            raise RuntimeError("graph replay at a step phase different from its capture")
        s._clock.fill_(float(s.time))
        _native.check(s._lib.cvlbm_graph_launch(self.handle, s._stream()), "cvlbm_graph_launch")
        for _ in range(self.nsteps):
            s.time += s.dt
        s.steps += self.nsteps
        s._stress_current = False

    def __del__(self) -> None:
        try:
            if self.handle:
                self.solver._lib.cvlbm_graph_destroy(self.handle)
        except Exception:
            pass


def relative_l2(error: np.ndarray, reference: np.ndarray, mask: np.ndarray) -> float:
    err, ref = np.asarray(error), np.asarray(reference)
    m = np.asarray(mask, dtype=bool)
    num = float(np.sqrt(np.sum(err[..., m] ** 2)))
    den = float(np.sqrt(np.sum(ref[..., m] ** 2)))
    return num / max(den, np.finfo(float).eps)


def constant_piola_params(material: WarpHyperelasticMaterial, F: np.ndarray):
    """Params for CURVED_VALUE_PIOLA_NORMAL from a constant F (reference :4485-4491)."""
    F4 = np.asarray(F, dtype=np.float64).reshape(2, 2)
    P = _first_piola_np(F4, material)
    return float(P[0, 0]), float(P[0, 1]), float(P[1, 0]), float(P[1, 1])


__all__ = [name for name in dir() if not name.startswith("__")]
