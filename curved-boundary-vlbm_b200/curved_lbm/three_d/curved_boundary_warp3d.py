"""Three-dimensional curved-boundary D3Q6x12 solver on active nodes (drop-in).

Same module path, names, constructor arguments, methods and errors as the
reference's ``curved_lbm.three_d.curved_boundary_warp3d`` (curved_lbm 1.0.0),
whose public class ``WarpCurvedBoundaryLBM3D`` is the sparse active-node
solver (:3852-4805).  The time step runs in hand-written sm_100a kernels
(``libcvlbm.so``) on PyTorch CUDA buffers.  Links whose three displacement
rows mix Dirichlet and Neumann kinds take the reference's component-wise
normal solve.  ``WarpCurvedBoundaryLBM3D`` is this sparse class (the
reference's dense 3-D class is not provided).
"""

from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Literal

import numpy as np

from .. import _native, _stamp
from .characteristic_stencil3d import MAX_CHARACTERISTIC_SAMPLES, build_characteristic_weights
from .geometry3d import (
    BOUNDARY_ID_INNER,
    BOUNDARY_ID_OUTER,
    DIRS3,
    MAX_BOUNDARY_IDS,
    MAX_LSQ_STENCIL,
    CurvedBoundaryGeometry3D,
    CurvedBoundarySpec3D,
    SphereDomain,
    _affine_neo_hooke_F_P_np,
    _basis_np,
    _build_sparse_tangent_lsq_weights,
    _kind_id,
    _solve_Fb_np,
    _sparse_tables_from_geometry,
    _value_np,
    constant_piola_params3d,
)
from .vector_nonlinear_elastic_warp3d import (
    BC_DIRICHLET,
    BC_NEUMANN,
    FQ,
    MATERIAL_NEO_HOOKE,
    NCOMP,
    PI,
    Q,
    SOURCE_CONSTANT,
    SOURCE_DAMPING,
    VALUE_AFFINE_VELOCITY,
    VALUE_CONSTANT,
    VALUE_SINE2_HOLD,
    VALUE_ZERO,
    WarpHyperelasticMaterial3D,
    _cofactor_np,
    _det3_np,
    _equilibrium_np,
    _first_piola_np,
    _source_np,
    _state_to_F_np,
    default_device,
    source_id,
    source_name,
)

CURVED3D_VALUE_ZERO = VALUE_ZERO
CURVED3D_VALUE_CONSTANT_VECTOR = VALUE_CONSTANT
CURVED3D_VALUE_AFFINE_VELOCITY = VALUE_AFFINE_VELOCITY
CURVED3D_VALUE_RAMP_VECTOR = 200
CURVED3D_VALUE_SINE2_HOLD_VECTOR = 204
CURVED3D_VALUE_PIOLA_NORMAL = 201
CURVED3D_VALUE_NORMAL_TRACTION = 202
CURVED3D_VALUE_SINE2_NORMAL_TRACTION = 203
CURVED3D_VALUE_AFFINE_NEO_HOOKE_PIOLA_NORMAL = 205
CURVED3D_VALUE_Z_PULL_TORSION_TRACTION = 206
CURVED3D_VALUE_Z_STRETCH_EXACT_TWIST_VELOCITY = 207
# Not in the reference: normal traction amp*min(t/ramp_time, 1)*n,
# params (amp, ramp_time).  Used by the linear-ramp shell workload.
CURVED3D_VALUE_LINEAR_NORMAL_TRACTION = 208

CURVED_VALUE_ZERO = CURVED3D_VALUE_ZERO
CURVED_VALUE_CONSTANT_VECTOR = CURVED3D_VALUE_CONSTANT_VECTOR
CURVED_VALUE_AFFINE_VELOCITY = CURVED3D_VALUE_AFFINE_VELOCITY
CURVED_VALUE_RAMP_VECTOR = CURVED3D_VALUE_RAMP_VECTOR
CURVED_VALUE_SINE2_HOLD_VECTOR = CURVED3D_VALUE_SINE2_HOLD_VECTOR
CURVED_VALUE_PIOLA_NORMAL = CURVED3D_VALUE_PIOLA_NORMAL
CURVED_VALUE_NORMAL_TRACTION = CURVED3D_VALUE_NORMAL_TRACTION
CURVED_VALUE_SINE2_NORMAL_TRACTION = CURVED3D_VALUE_SINE2_NORMAL_TRACTION
CURVED_VALUE_AFFINE_NEO_HOOKE_PIOLA_NORMAL = CURVED3D_VALUE_AFFINE_NEO_HOOKE_PIOLA_NORMAL
CURVED_VALUE_Z_PULL_TORSION_TRACTION = CURVED3D_VALUE_Z_PULL_TORSION_TRACTION
CURVED_VALUE_Z_STRETCH_EXACT_TWIST_VELOCITY = CURVED3D_VALUE_Z_STRETCH_EXACT_TWIST_VELOCITY

BOUNDARY_RECON_BFL = 0
BOUNDARY_RECON_HALF_WAY = 1
BOUNDARY_RECON_COMPAT_BFL = 2
BOUNDARY_RECON_LOCAL_F = 3
BOUNDARY_RECON_LOCAL_F_BFL = 4
NORMAL_JACOBIAN_FINITE_DIFFERENCE = 0
NORMAL_JACOBIAN_ACOUSTIC = 1
NORMAL_SOLVER_ENERGY = 2

BoundaryReconstruction = Literal["bfl", "halfway", "compat_bfl", "local_f", "local_f_bfl"]


def neumann_solver_name(name, material) -> str:
    """Reference :112-127; honours XLB_NEUMANN_SOLVER."""
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
    value = os.environ.get("XLB_NORMAL_JACOBIAN", "acoustic") if name is None else str(name)
    key = value.strip().lower().replace("-", "_")
    if key in ("finite_difference", "finite", "fd"):
        return NORMAL_JACOBIAN_FINITE_DIFFERENCE
    if key in ("acoustic", "acoustic_tensor", "analytic", "analytical"):
        return NORMAL_JACOBIAN_ACOUSTIC
    raise ValueError(f"unsupported normal Jacobian mode: {value!r}")


def normal_jacobian_name(mode: int) -> str:
    return {0: "finite_difference", 1: "acoustic"}.get(int(mode), f"unknown({mode})")


def _normal_jacobian_for_material(material, mode) -> int:
    if mode is None and material.model == "sph_neo_hooke":
        return NORMAL_JACOBIAN_FINITE_DIFFERENCE
    return normal_jacobian_id(mode)


def _recon_id(k: str) -> int:
    table = {"bfl": 0, "bouzidi": 0, "bouzidi_firdaouss_lallemand": 0, "halfway": 1,
             "half_way": 1, "half-way": 1, "compat_bfl": 2, "local_f": 3, "fully_local": 3,
             "local_f_bfl": 4, "single_history": 4}
    if k not in table:
        raise ValueError(f"unsupported boundary_reconstruction: {k}")
    return table[k]


def _recon_name(rid: int) -> str:
    return {0: "bfl", 1: "halfway", 2: "compat_bfl", 3: "local_f", 4: "local_f_bfl"}.get(
        int(rid), f"unknown({rid})")


WAVE_CHUNK = 128  # nodes per work item of the wavefront kernel (its block size)


WAVE_LAGS = (1, 3)  # planes by which the sweep and the collide trail the moments


def _wave_tables3(active_i, nx: int, lags=WAVE_LAGS):
    """Work items of the wavefront node kernel (node_variant 3/4), in ticket order.

    The active ids run through the x-planes in order; each plane is cut into
    chunks of WAVE_CHUNK nodes.  For w = 0, 1, ... the items are the moments
    chunks of plane w, the sweep chunks of plane w-ls and the collide chunks
    of plane w-lc, (ls, lc) = `lags` with ls >= 1 and lc >= ls + 2: every
    item depends only on items before it (sweep of plane i on the moments of
    i-1..i+1, collide of plane i on the sweeps of i-2..i+2); larger lags wait
    less and keep more planes in flight.  Returns (items [n, 4] int32: stage,
    plane, first id, end id; chunks per plane [nx] int32).
    """
    ls, lc = int(lags[0]), int(lags[1])
    if ls < 1 or lc < ls + 2:
        raise ValueError(f"wave lags {lags} break the item order (need ls >= 1, lc >= ls + 2)")
    ai = np.asarray(active_i, dtype=np.int64)
    start = np.searchsorted(ai, np.arange(nx + 1), side="left")
    counts = np.diff(start)
    chunks = ((counts + WAVE_CHUNK - 1) // WAVE_CHUNK).astype(np.int32)
    rows = []
    for w in range(nx + lc):
        for stage, plane in ((0, w), (1, w - ls), (2, w - lc)):
            if 0 <= plane < nx:
                a, b = int(start[plane]), int(start[plane + 1])
                for c0 in range(a, b, WAVE_CHUNK):
                    rows.append((stage, plane, c0, min(c0 + WAVE_CHUNK, b)))
    items = np.asarray(rows, dtype=np.int32).reshape(-1, 4)
    return np.ascontiguousarray(items), chunks


def _fused_tables3(tables, link_q, comp_kind, stencil, n_active):
    """Tables of the fused 3-D step, or None when the links do not allow it.

    * need_slot: for each active node whose post-step U some cut link reads
      (the cut node, its upstream node and the characteristic stencil) its
      row in the U_need buffer, -1 elsewhere; char_slot: the characteristic
      stencil's node ids mapped to those rows;
    * partner: for link (p, q_out) whose upstream node p - c_q is not active,
      the link (p, q_in) at the same node, whose stored outgoing population is
      this link's post-collision f[q_in](p); -1 when the upstream is active;
    * order: links with a Neumann row first, so the warps of the
      one-thread-per-link kernels take the same branches.
    """
    link_p = np.asarray(tables["link_p"], dtype=np.int64)
    up = np.asarray(tables["link_upstream"], dtype=np.int64)
    q = np.asarray(link_q, dtype=np.int64)
    nl = link_p.size
    need = np.zeros(n_active, dtype=bool)
    if nl:
        need[link_p] = True
        need[up[up >= 0]] = True
    idx = None
    if stencil is not None:
        idx = np.asarray(stencil["indices"], dtype=np.int64)
        need[idx[idx >= 0]] = True
    need_slot = np.full(n_active, -1, dtype=np.int32)
    need_slot[need] = np.arange(int(need.sum()), dtype=np.int32)
    char_slot = None
    if idx is not None:
        char_slot = np.where(idx >= 0, need_slot[np.maximum(idx, 0)], -1).astype(np.int32)
    partner = np.full(nl, -1, dtype=np.int32)
    if nl:
        key = link_p * 6 + q
        pos = {int(k): e for e, k in enumerate(key)}
        for e in np.flatnonzero(up < 0):
            qi = (int(q[e]) + 3) % 6
            j = pos.get(int(link_p[e]) * 6 + qi, -1)
            if j < 0:
                return None
            partner[e] = j
    neumann = (np.any(np.asarray(comp_kind).reshape(3, -1) == BC_NEUMANN, axis=0) if nl
               else np.zeros(0, bool))
    order = np.concatenate([np.flatnonzero(neumann), np.flatnonzero(~neumann)]).astype(np.int32)
    return need_slot, char_slot, partner, np.ascontiguousarray(order)


def _node_link_csr(link_node: np.ndarray, n_nodes: int):
    valid = link_node >= 0
    ids = np.flatnonzero(valid).astype(np.int32)
    nodes = link_node[valid]
    order = ids[np.argsort(nodes, kind="stable")]
    counts = np.bincount(nodes, minlength=n_nodes) if nodes.size else np.zeros(n_nodes, np.int64)
    start = np.zeros(n_nodes + 1, dtype=np.int32)
    np.cumsum(counts, out=start[1:])
    return start, np.ascontiguousarray(order.astype(np.int32))


class WarpSparseCurvedBoundaryLBM3D:
    """Active-node sparse curved 3-D solver on sm_100a (reference :3852-4802).

    Device buffers (torch, float64): ``f0, f1`` (72, n_active), ``U``
    (12, n_active), ``u, u_star`` (3, n_active); per-link boundary data
    ``link_Fb, link_Pb`` (9, n_links), ``link_bv`` (3, n_links),
    ``char_state`` (4, 12, n_links).
    """

    def __init__(self, geometry: CurvedBoundaryGeometry3D, *, material: WarpHyperelasticMaterial3D,
                 boundary: CurvedBoundarySpec3D, lattice_speed: float = 5.0,
                 collision_omega: float = 1.8, boundary_reconstruction: str = "bfl",
                 device: str | None = None, check_linearized_cfl: bool = True,
                 jacobian_floor: float = 1e-12, source_mode: str = "none",
                 source_vector: tuple = (0.0,) * NCOMP, damping_gamma: float = 0.0,
                 compatibility_projection_interval: int = 0,
                 compatibility_projection_iterations: int = 160,
                 compatibility_projection_relax: float = 0.85,
                 compatibility_projection_weight: float = 20.0,
                 compatibility_projection_repair_F: bool = False,
                 compatibility_projection_repair_F_band_width: int = -1,
                 compatibility_projection_repair_F_blend: float = 1.0,
                 compatibility_projection_boundary_id: int = -1,
                 local_displacement_interval: int = 0, local_displacement_sweeps: int = 1,
                 local_displacement_relax: float = 0.85,
                 local_displacement_boundary_weight: float = 20.0,
                 local_displacement_boundary_id: int = -1, local_compatibility_interval: int = 0,
                 local_compatibility_blend: float = 0.1, normal_jacobian: str | None = None,
                 neumann_solver: str | None = None, characteristic_stencil: dict | None = None):
        """`characteristic_stencil` (not in the reference): precomputed
        local_f stencil tables in build_characteristic_weights' layout, used
        instead of building them on the device (e.g. to run on the exact
        tables of another builder)."""
        import torch

        self.geometry = geometry
        self.nx, self.ny, self.nz = geometry.nx, geometry.ny, geometry.nz
        self.length_x, self.length_y, self.length_z = (geometry.length_x, geometry.length_y,
                                                       geometry.length_z)
        self.dx, self.dy, self.dz = geometry.dx, geometry.dy, geometry.dz
        self.material = material
        self.boundary = boundary
        self.lattice_speed = float(lattice_speed)
        self.collision_omega = float(collision_omega)
        if not (0.0 < self.collision_omega <= 2.0):
            raise ValueError("collision_omega must be in (0,2]")
        self.boundary_reconstruction = _recon_id(boundary_reconstruction)
        self.boundary_reconstruction_name = _recon_name(self.boundary_reconstruction)
        self.normal_jacobian = _normal_jacobian_for_material(material, normal_jacobian)
        self.normal_jacobian_name = normal_jacobian_name(self.normal_jacobian)
        self.neumann_solver_name = neumann_solver_name(neumann_solver, material)
        self._normal_solver_mode = (NORMAL_SOLVER_ENERGY if self.neumann_solver_name == "energy"
                                    else self.normal_jacobian)
        self.dt = self.dx / self.lattice_speed
        self.time = 0.0
        self.steps = 0
        self.shape = (self.nx, self.ny, self.nz)
        self.jacobian_floor = float(jacobian_floor)
        if check_linearized_cfl and material.linearized_stability_ratio(self.lattice_speed) >= 1.0:
            raise ValueError("linearized D3Q6 stability ratio must be below one")
        self.source_mode = source_id(source_mode)
        self.source_params = np.zeros(NCOMP)
        if self.source_mode == SOURCE_CONSTANT:
            for i, v in enumerate(tuple(source_vector)[:NCOMP]):
                self.source_params[i] = float(v)
        elif self.source_mode == SOURCE_DAMPING:
            self.source_params[0] = float(damping_gamma)
        if int(compatibility_projection_interval) != 0:
            raise ValueError("the fully-local solver forbids compatibility_projection_interval != 0")
        self.compatibility_projection_interval = 0
        self.compatibility_projection_iterations = int(max(1, compatibility_projection_iterations))
        self.compatibility_projection_relax = float(compatibility_projection_relax)
        self.compatibility_projection_weight = float(compatibility_projection_weight)
        self.compatibility_projection_repair_F = False
        self.compatibility_projection_repair_F_band_width = int(compatibility_projection_repair_F_band_width)
        self.compatibility_projection_repair_F_blend = float(compatibility_projection_repair_F_blend)
        self.compatibility_projection_boundary_id = int(compatibility_projection_boundary_id)
        self._compatibility_projector = None
        self.local_displacement_interval = int(max(0, local_displacement_interval))
        self.local_displacement_sweeps = int(local_displacement_sweeps)
        self.local_displacement_relax = float(local_displacement_relax)
        self.local_displacement_boundary_weight = float(local_displacement_boundary_weight)
        self.local_displacement_boundary_id = int(local_displacement_boundary_id)
        self.local_compatibility_interval = int(max(0, local_compatibility_interval))
        self.local_compatibility_blend = float(local_compatibility_blend)
        if not (1 <= self.local_displacement_sweeps <= 8):
            raise ValueError("local_displacement_sweeps must be in [1,8]")
        if not (0.0 <= self.local_displacement_relax <= 1.0):
            raise ValueError("local_displacement_relax must be in [0,1]")
        if self.local_displacement_boundary_weight < 0.0:
            raise ValueError("local_displacement_boundary_weight must be non-negative")
        if not (0.0 <= self.local_compatibility_blend <= 1.0):
            raise ValueError("local_compatibility_blend must be in [0,1]")
        self._x_dense = self._y_dense = self._z_dense = None
        self.active_np = np.ascontiguousarray(geometry.active.astype(np.int32))
        tables = _sparse_tables_from_geometry(geometry)
        self.active_i, self.active_j, self.active_k = (tables["active_i"], tables["active_j"],
                                                       tables["active_k"])
        self.active_id_np = tables["active_id"]
        self.n_active = int(self.active_i.size)
        self.n_nodes = self.n_active
        nl = int(geometry.n_links)
        self.tangent_lsq_active = self.boundary_reconstruction == BOUNDARY_RECON_COMPAT_BFL
        if self.tangent_lsq_active:
            lsq = _build_sparse_tangent_lsq_weights(geometry, tables)
        else:
            lsq = {"lsq_p": np.zeros((nl, MAX_LSQ_STENCIL), np.int32),
                   "lsq_wt1": np.zeros((nl, MAX_LSQ_STENCIL)),
                   "lsq_wt2": np.zeros((nl, MAX_LSQ_STENCIL)), "lsq_valid": np.zeros(nl, np.int32)}
        self.lsq_valid_np = lsq["lsq_valid"]
        self.kind_by_id, self.mode_by_id, self.params_by_id = boundary.tables(MAX_BOUNDARY_IDS)
        self.component_kind_by_id = boundary.component_kind_table(MAX_BOUNDARY_IDS)
        link_ids = np.asarray(geometry.link_boundary_id, dtype=np.int32)
        clipped = np.clip(link_ids, 0, MAX_BOUNDARY_IDS - 1)
        ck = self.component_kind_by_id[:, clipped]
        self._has_neumann_cut_links = bool(link_ids.size and np.any(ck == BC_NEUMANN))
        self.characteristic_stencil = None
        if self.boundary_reconstruction == BOUNDARY_RECON_LOCAL_F and self._has_neumann_cut_links:
            if characteristic_stencil is not None:
                cs = characteristic_stencil
                want = (MAX_CHARACTERISTIC_SAMPLES, int(geometry.n_links))
                if np.shape(cs["indices"]) != want or np.shape(cs["weights"]) != (4,) + want:
                    raise ValueError("characteristic_stencil does not match this geometry")
                self.characteristic_stencil = {
                    "indices": np.ascontiguousarray(cs["indices"], dtype=np.int32),
                    "weights": np.ascontiguousarray(cs["weights"], dtype=np.float64),
                    "probe_modes": np.asarray(cs.get("probe_modes", np.zeros(want[1])),
                                              dtype=np.int32)}
            else:
                self.characteristic_stencil = build_characteristic_weights(
                    geometry, tables, link_mask=np.any(ck == BC_NEUMANN, axis=0),
                    device=str(device or default_device()))
        self.memory = None

        self.device = str(device or default_device())
        self._tdev = _native.torch_device(self.device)
        self._lib = _native.load()
        dev, f64, i32 = self._tdev, torch.float64, torch.int32

        def dev_i(a):
            return torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)

        def dev_f(a):
            return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)

        start, order = _node_link_csr(tables["link_p"].astype(np.int64), self.n_active)
        t = {
            "active_i": dev_i(self.active_i), "active_j": dev_i(self.active_j),
            "active_k": dev_i(self.active_k), "neighbor": dev_i(tables["neighbor"]),
            "link_p": dev_i(tables["link_p"]), "link_up": dev_i(tables["link_upstream"]),
            "link_q": dev_i(geometry.link_q), "link_bid": dev_i(clipped),
            "link_eta": dev_f(geometry.link_eta), "link_xb": dev_f(geometry.link_xb),
            "link_yb": dev_f(geometry.link_yb), "link_zb": dev_f(geometry.link_zb),
            "link_nx": dev_f(geometry.link_nx), "link_ny": dev_f(geometry.link_ny),
            "link_nz": dev_f(geometry.link_nz), "lsq_p": dev_i(lsq["lsq_p"]),
            "lsq_wt1": dev_f(lsq["lsq_wt1"]), "lsq_wt2": dev_f(lsq["lsq_wt2"]),
            "lsq_valid": dev_i(lsq["lsq_valid"]), "node_link_start": dev_i(start),
            "node_link_list": dev_i(order), "bc_kind": dev_i(self.kind_by_id),
            "bc_mode": dev_i(self.mode_by_id), "bc_comp_kind": dev_i(self.component_kind_by_id),
            "bc_params": dev_f(self.params_by_id),
        }
        if self.characteristic_stencil is not None:
            t["char_idx"] = dev_i(self.characteristic_stencil["indices"])
            t["char_w"] = dev_f(self.characteristic_stencil["weights"])
        fused = _fused_tables3(tables, geometry.link_q, ck, self.characteristic_stencil,
                               self.n_active)
        self._n_need = 0
        if fused is not None:
            need_slot, char_slot, partner, order = fused
            self._n_need = int(need_slot.max()) + 1 if need_slot.size else 0
            t["need_slot"] = dev_i(need_slot)
            if char_slot is not None:
                t["char_slot"] = dev_i(char_slot)
                # link-major copies for the fused gather: a link's slots and,
                # per sample, its four weights side by side
                t["char_slot_lm"] = t["char_slot"].view(-1, nl).t().contiguous()
                t["char_w_lm"] = t["char_w"].view(4, -1, nl).permute(2, 1, 0).contiguous()
            t["link_partner"] = dev_i(partner)
            t["link_order"] = dev_i(order)
        link_nodes = np.unique(np.asarray(tables["link_p"], dtype=np.int64))
        self._n_link_nodes = int(link_nodes.size)
        if link_nodes.size:
            t["link_nodes"] = dev_i(link_nodes)
        self._active_i_np = np.asarray(tables["active_i"])
        items, chunks = _wave_tables3(self._active_i_np, self.nx)
        self._n_wave_items = int(items.shape[0])
        t["wave_items"] = dev_i(items.reshape(-1))
        t["wave_plane_chunks"] = dev_i(chunks)
        self._wave_sync = torch.zeros(2 + 3 * self.nx, dtype=i32, device=dev)
        self._tables = t
        self.neighbor = t["neighbor"]
        self.link_p = t["link_p"]
        self.link_upstream = t["link_up"]
        self.dynamic_traction_override_enabled = torch.zeros(nl, dtype=i32, device=dev)
        self.dynamic_traction_override = torch.zeros((3, nl), dtype=f64, device=dev)
        n = self.n_active
        self.f0 = torch.zeros((FQ, n), dtype=f64, device=dev)
        self.f1 = torch.zeros_like(self.f0)
        self.u = torch.zeros((3, n), dtype=f64, device=dev)
        self.u_star = torch.zeros_like(self.u)
        self.U = torch.zeros((NCOMP, n), dtype=f64, device=dev)
        self.u_local_next = torch.zeros_like(self.u)
        self.link_kind = torch.zeros(nl, dtype=i32, device=dev)
        self.link_component_kind = torch.zeros((3, nl), dtype=i32, device=dev)
        self.link_bv = torch.zeros((3, nl), dtype=f64, device=dev)
        self.link_Fb = torch.zeros((9, nl), dtype=f64, device=dev)
        self.link_Pb = torch.zeros((9, nl), dtype=f64, device=dev)
        self.char_state = (torch.zeros((4, NCOMP, nl), dtype=f64, device=dev)
                           if self.characteristic_stencil is not None
                           else torch.zeros((1, 1, 1), dtype=f64, device=dev))
        self.invalid = torch.zeros(1, dtype=i32, device=dev)
        self._clock = torch.zeros(1, dtype=f64, device=dev)
        self.link_scratch = torch.zeros(max(1, 12 * nl), dtype=f64, device=dev)
        self.U_need = torch.zeros(max(1, 12 * self._n_need), dtype=f64, device=dev)
        self.source_params_wp = self.source_params.copy()
        self._problem = self._make_problem()
        self.initialize_identity()

    # -- native plumbing ---------------------------------------------------
    def _make_problem(self) -> _native.Problem3D:
        m = self.material
        p = _native.Problem3D()
        p.n_active, p.n_links = self.n_active, int(self.geometry.n_links)
        p.nx, p.ny, p.nz = self.nx, self.ny, self.nz
        p.recon = int(self.boundary_reconstruction)
        p.normal_solver = int(self._normal_solver_mode)
        p.source_mode = int(self.source_mode)
        p.has_char = int(self.characteristic_stencil is not None)
        p.has_tangent_lsq = int(self.tangent_lsq_active)
        p.disp_interval = self.local_displacement_interval
        p.disp_sweeps = self.local_displacement_sweeps
        p.disp_bid = self.local_displacement_boundary_id
        p.rep_interval = self.local_compatibility_interval
        p.dx, p.dy, p.dz, p.dt = self.dx, self.dy, self.dz, self.dt
        p.omega, p.c = self.collision_omega, self.lattice_speed
        for i in range(NCOMP):
            p.source[i] = float(self.source_params[i])
        p.mat = _native.Material(int(m.id), 0, float(m.lam), float(m.mu), float(m.param0),
                                 float(m.param1), float(m.param2), self.jacobian_floor)
        p.relax = self.local_displacement_relax
        p.weight = self.local_displacement_boundary_weight
        p.blend = self.local_compatibility_blend
        for name, tensor in self._tables.items():
            setattr(p, name, _native.ptr(tensor))
        p.n_need = self._n_need
        p.n_link_nodes = self._n_link_nodes
        p.n_wave_items, p.n_planes = self._n_wave_items, self.nx
        p.overlap = 0  # measured slower on shell192: the link kernels are throughput-bound
        p.dyn_enabled = _native.ptr(self.dynamic_traction_override_enabled)
        p.dyn_traction = _native.ptr(self.dynamic_traction_override)
        return p

    def _fields(self) -> _native.Fields3D:
        fl = _native.Fields3D()
        has_char = self.characteristic_stencil is not None
        for name, tensor in (("f0", self.f0), ("f1", self.f1), ("U", self.U), ("u", self.u),
                             ("u_next", self.u_local_next), ("u_star", self.u_star),
                             ("link_kind", self.link_kind),
                             ("link_comp_kind", self.link_component_kind),
                             ("link_bv", self.link_bv), ("link_Fb", self.link_Fb),
                             ("link_Pb", self.link_Pb),
                             ("char_state", self.char_state if has_char else None),
                             ("invalid", self.invalid), ("clock", self._clock),
                             ("link_scratch", self.link_scratch), ("U_need", self.U_need),
                             ("wave_sync", self._wave_sync)):
            setattr(fl, name, _native.ptr(tensor))
        return fl

    def _stream(self) -> int:
        return _native.stream_ptr(self._tdev)

    # -- dynamic traction (reference :4115-4174) ----------------------------
    def _validate_dynamic_traction_override(self, enabled, traction) -> None:
        import torch

        nl = self.geometry.n_links
        if tuple(enabled.shape) != (nl,):
            raise ValueError(f"dynamic traction enable mask must have shape {(nl,)}")
        if tuple(traction.shape) != (3, nl):
            raise ValueError(f"dynamic traction values must have shape {(3, nl)}")
        if enabled.dtype != torch.int32:
            raise TypeError("dynamic traction enable mask must use int32")
        if traction.dtype != torch.float64:
            raise TypeError("dynamic traction values must use float64")
        if enabled.device != self._tdev or traction.device != self._tdev:
            raise ValueError(f"dynamic traction buffers must reside on {self._tdev}")

    def bind_dynamic_traction_override(self, enabled, traction) -> None:
        """Bind externally owned device buffers without copying them."""
        self._validate_dynamic_traction_override(enabled, traction)
        self.dynamic_traction_override_enabled = enabled.contiguous()
        self.dynamic_traction_override = traction.contiguous()
        self._problem.dyn_enabled = _native.ptr(self.dynamic_traction_override_enabled)
        self._problem.dyn_traction = _native.ptr(self.dynamic_traction_override)

    def update_dynamic_traction_override(self, *, enabled=None, traction=None) -> None:
        import torch

        nl = self.geometry.n_links
        if enabled is not None:
            arr = torch.as_tensor(np.asarray(enabled, dtype=np.int32) if isinstance(enabled, np.ndarray)
                                  else enabled)
            if tuple(arr.shape) != (nl,):
                raise ValueError(f"dynamic traction enable mask must have shape {(nl,)}")
            self.dynamic_traction_override_enabled.copy_(arr.to(self._tdev, torch.int32))
        if traction is not None:
            arr = torch.as_tensor(np.asarray(traction, dtype=np.float64)
                                  if isinstance(traction, np.ndarray) else traction)
            if tuple(arr.shape) != (3, nl):
                raise ValueError(f"dynamic traction values must have shape {(3, nl)}")
            self.dynamic_traction_override.copy_(arr.to(self._tdev, torch.float64))

    def clear_dynamic_traction_override(self) -> None:
        self.dynamic_traction_override_enabled.zero_()

    # -- geometry helpers ----------------------------------------------------
    def _build_dense_coordinates(self) -> None:
        if self._x_dense is None:
            xs = (np.arange(self.nx) + 0.5) * self.dx
            ys = (np.arange(self.ny) + 0.5) * self.dy
            zs = (np.arange(self.nz) + 0.5) * self.dz
            self._x_dense, self._y_dense, self._z_dense = np.meshgrid(xs, ys, zs, indexing="ij")

    @property
    def x(self):
        self._build_dense_coordinates()
        return self._x_dense

    @property
    def y(self):
        self._build_dense_coordinates()
        return self._y_dense

    @property
    def z(self):
        self._build_dense_coordinates()
        return self._z_dense

    def active_indices(self):
        return self.active_i.copy(), self.active_j.copy(), self.active_k.copy()

    def active_coordinates(self):
        return ((self.active_i.astype(np.float64) + 0.5) * self.dx,
                (self.active_j.astype(np.float64) + 0.5) * self.dy,
                (self.active_k.astype(np.float64) + 0.5) * self.dz)

    def memory_estimate_bytes(self) -> dict:
        nl = self.geometry.n_links
        return {"populations": int(2 * FQ * self.n_active * 8),
                "fields": int((NCOMP + 3 + 3 + 3 + 3 + 3) * self.n_active * 8),
                "connectivity": int((Q * self.n_active + 2 * nl) * 4),
                "link_data": int((1 + 3 + 9 + 9 + 3) * nl * 8 + nl * 4)}

    def _active_from_dense(self, arr, ncomp, name):
        arr = np.asarray(arr, dtype=np.float64)
        if arr.shape == (ncomp, self.n_active):
            return np.ascontiguousarray(arr)
        if arr.shape != (ncomp, self.nx, self.ny, self.nz):
            raise ValueError(
                f"{name} must have shape {(ncomp, self.nx, self.ny, self.nz)} or {(ncomp, self.n_active)}")
        return np.ascontiguousarray(arr[:, self.active_np.astype(bool)])

    def _scatter_to_dense(self, values, ncomp, *, identity_U=False):
        out = np.zeros((ncomp, self.nx, self.ny, self.nz), dtype=np.float64)
        if identity_U and ncomp == NCOMP:
            out[3] = out[7] = out[11] = 1.0
        out[:, self.active_i, self.active_j, self.active_k] = values
        return out

    def _source_active_np(self, U):
        out = np.zeros_like(U)
        if self.source_mode == SOURCE_CONSTANT:
            out[:] = self.source_params[:NCOMP, None]
        elif self.source_mode == SOURCE_DAMPING:
            for a in range(3):
                out[a] = -self.source_params[0] * U[a]
        return out

    # -- initialisation (reference :4207-4279) --------------------------------
    def initialize_identity(self, *, init_order: int = 1):
        U = np.zeros((NCOMP, self.n_active))
        U[3] = U[7] = U[11] = 1.0
        self._initialize_from_active(U, np.zeros((3, self.n_active)), init_order=init_order)

    def initialize_from_numpy(self, *, U, displacement=None, init_order: int = 1,
                              apply_initial_boundaries: bool = True,
                              initial_boundary_time: float = 0.0):
        Ua = self._active_from_dense(U, NCOMP, "U")
        da = (np.zeros((3, self.n_active)) if displacement is None
              else self._active_from_dense(displacement, 3, "displacement"))
        self._initialize_from_active(Ua, da, init_order=init_order,
                                     apply_initial_boundaries=apply_initial_boundaries,
                                     initial_boundary_time=initial_boundary_time)

    def _initialize_from_active(self, U_active, disp_active, *, init_order=1,
                                apply_initial_boundaries=True, initial_boundary_time=0.0):
        import torch

        if init_order != 1:
            raise ValueError(
                "sparse 3-D curved solver currently supports init_order=1; use dense class for "
                "higher-order initialization")
        f = _equilibrium_np(U_active, self.material, self.lattice_speed)
        f -= 0.5 * self.dt / float(Q) * self._source_active_np(U_active)[None, ...]
        dev = self._tdev
        self.f0.copy_(torch.as_tensor(np.ascontiguousarray(f.reshape(FQ, self.n_active)), device=dev))
        self.f1.zero_()
        us0 = np.ascontiguousarray(disp_active - 0.5 * self.dt * U_active[:3])
        self.u_star.copy_(torch.as_tensor(us0, device=dev))
        self.time = 0.0
        self.steps = 0
        self.refresh_current()
        if apply_initial_boundaries:
            self.apply_boundary_reconstruction(initial_boundary_time, in_place=True)
            self.refresh_current()
            disp = torch.as_tensor(np.ascontiguousarray(disp_active, dtype=np.float64), device=dev)
            _native.check(self._lib.cvlbm3d_set_ustar(self._problem, self._fields(),
                                                      _native.ptr(disp), self._stream()),
                          "cvlbm3d_set_ustar")
            self.refresh_current()

    # -- boundary ----------------------------------------------------------
    def apply_boundary_reconstruction(self, t: float, *, in_place: bool = False):
        """Reference :4339-4399."""
        if self.geometry.n_links == 0:
            return
        _native.check(self._lib.cvlbm3d_apply_boundary(self._problem, self._fields(), float(t),
                                                       int(bool(in_place)), self._stream()),
                      "cvlbm3d_apply_boundary")

    def configure_compatibility_projection(self, *, interval=1, iterations=160, relax=0.85,
                                           weight=20.0, repair_F=False, repair_F_band_width=-1,
                                           repair_F_blend=1.0, boundary_id=-1) -> None:
        if int(interval) != 0 or bool(repair_F):
            raise ValueError("global compatibility projection is not available in the fully-local solver")

    def project_compatible_displacement(self, *, iterations=None, repair_F=None) -> None:
        raise RuntimeError("global compatibility projection is disabled by design")

    def _compatibility_projection_due(self) -> bool:
        return False

    def _local_displacement_due(self) -> bool:
        return self.local_displacement_interval > 0 and self.steps % self.local_displacement_interval == 0

    def _local_compatibility_due(self) -> bool:
        return self.local_compatibility_interval > 0 and self.steps % self.local_compatibility_interval == 0

    # -- time stepping -------------------------------------------------------
    def run(self, nsteps: int) -> None:
        """Advance ``nsteps`` steps in one native call (no host sync)."""
        nsteps = int(nsteps)
        if nsteps <= 0:
            return
        _native.check(self._lib.cvlbm3d_run(self._problem, self._fields(), float(self.time),
                                            int(self.steps), nsteps, 0, self._stream()),
                      "cvlbm3d_run")
        if nsteps % 2 == 1:
            self.f0, self.f1 = self.f1, self.f0
        for _ in range(nsteps):
            self.time += self.dt
        self.steps += nsteps

    # fused collide kernel: 0 one thread per node (128 registers), 1 six warps
    # per 32 nodes (shared memory), 2 one thread per node (168 registers)
    NODE_VARIANTS = (0, 1, 2, 3, 4)

    @property
    def overlap_links(self) -> bool:
        """Run the next step's moments of the nodes without a cut link on a
        second stream while the link kernels run (fused step with a sweep every
        step; results are identical either way).  Off by default: the 3-D link
        kernels are bound by memory throughput, so the overlapped moments only
        compete with them (shell192: 2.01 ms per step against 1.91 ms)."""
        return bool(self._problem.overlap)

    @overlap_links.setter
    def overlap_links(self, on: bool) -> None:
        self._problem.overlap = int(bool(on))

    @property
    def node_variant(self) -> int:
        return int(self._problem.node_variant)

    def _select_variant(self, variant: int) -> None:
        """Pick the fused collide kernel (results are identical; speed differs)."""
        if int(variant) not in self.NODE_VARIANTS:
            raise ValueError(f"fused collide variant {variant} does not exist")
        self._problem.node_variant = int(variant)

    def _set_wave_lags(self, lags) -> None:
        """Rebuild the wavefront item order with other stage lags (same results)."""
        import torch

        items, _ = _wave_tables3(self._active_i_np, self.nx, lags)
        self._tables["wave_items"] = torch.as_tensor(items.reshape(-1), device=self._tdev)
        self._problem.wave_items = _native.ptr(self._tables["wave_items"])

    def autotune(self, steps: int = 10, variants=None) -> dict:
        """Time every fused collide variant on this problem; keep the fastest.

        Runs on a copy of the state that is restored afterwards, so the
        solution is unchanged.  Returns {variant: us/step}.
        """
        import torch

        saved = (self.f0.clone(), self.f1.clone(), self.u_star.clone(), self.U.clone(),
                 self.u.clone(), self.u_local_next.clone(), self.time, self.steps)
        times = {}
        for v in (variants if variants is not None else self.NODE_VARIANTS):
            self._select_variant(v)
            self.run(2)
            torch.cuda.synchronize(self._tdev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self.run(steps)
            e1.record()
            e1.synchronize()
            times[v] = e0.elapsed_time(e1) * 1e3 / steps
            for dst, src in zip((self.f0, self.f1, self.u_star, self.U, self.u,
                                 self.u_local_next), saved[:6]):
                dst.copy_(src)
            self.time, self.steps = saved[6], saved[7]
        self._select_variant(min(times, key=times.get))
        return times

    def step(self):
        """Reference :4549-4589."""
        self.run(1)

    def capture_graph(self, nsteps: int):
        return _Graph3D(self, int(nsteps))

    def refresh_current(self):
        """Reference :4401-4424."""
        _native.check(self._lib.cvlbm3d_refresh(self._problem, self._fields(), self._stream()),
                      "cvlbm3d_refresh")

    def run_until(self, t_end: float):
        """Reference :4591-4595."""
        import torch

        n = 0
        tt = self.time
        while tt < float(t_end) - 0.5 * self.dt:
            tt += self.dt
            n += 1
        self.run(n)
        self.refresh_current()
        torch.cuda.synchronize(self._tdev)

    # -- outputs (reference :4597-4769) ---------------------------------------
    def _host(self, tensor) -> np.ndarray:
        import torch

        torch.cuda.synchronize(self._tdev)
        return tensor.detach().cpu().numpy()

    def active_mask(self):
        return self.active_np.astype(bool)

    def active_system_state(self):
        return self._host(self.U)

    def active_displacement(self):
        return self._host(self.u)

    def active_ustar(self):
        return self._host(self.u_star)

    def active_populations(self):
        return self._host(self.f0)

    def active_deformation_gradient(self):
        return _state_to_F_np(self.active_system_state())

    def active_deformation_jacobian(self):
        return _det3_np(self.active_deformation_gradient())

    def active_piola(self):
        return _first_piola_np(self.active_deformation_gradient(), self.material)

    def active_sigma(self):
        F = self.active_deformation_gradient()
        P = _first_piola_np(F, self.material)
        J = np.maximum(_det3_np(F), self.jacobian_floor)
        return np.einsum("ia...,ja...->ij...", P, F) / J

    def numpy_field(self, name):
        if name == "U":
            return self._scatter_to_dense(self._host(self.U), NCOMP, identity_U=True)
        if name in ("u", "u_star"):
            return self._scatter_to_dense(self._host(getattr(self, name)), 3)
        if name in ("f0", "f1"):
            return self._scatter_to_dense(self._host(getattr(self, name)), FQ)
        if name in ("P", "sigma"):
            U = self._host(self.U)
            F = U[3:12].reshape(3, 3, self.n_active)
            P = _first_piola_np(F, self.material)
            if name == "P":
                return self._scatter_to_dense(P.reshape(9, self.n_active), 9)
            J = np.maximum(_det3_np(F), self.jacobian_floor)
            sigma = np.einsum("ia...,ja...->ij...", P, F) / J
            return self._scatter_to_dense(sigma.reshape(9, self.n_active), 9)
        raise AttributeError(name)

    def system_state(self):
        return self.numpy_field("U")

    def displacement(self):
        return self.numpy_field("u")

    def deformation_gradient(self):
        return _state_to_F_np(self.system_state())

    def deformation_jacobian(self):
        return _det3_np(self.deformation_gradient())

    def invalid_state(self):
        U = self._host(self.U)
        F = U[3:12].reshape(3, 3, self.n_active)
        return (int(self._host(self.invalid)[0]) != 0 or not np.isfinite(U).all()
                or not np.all(_det3_np(F) > 0))

    def summary(self):
        """The field reductions (max |u|, max |v|, min / max J, finite) run on
        the device (cvlbm_field_summary)."""
        self.refresh_current()
        red = _native.field_summary(self._lib, 3, self.n_active, self.U, self.u, None,
                                    self._tdev)
        mem = self.memory_estimate_bytes()
        drad = int(self.local_displacement_sweeps) if self.local_displacement_interval > 0 else 0
        crad = drad + 2 if self.local_compatibility_interval > 0 else drad
        ck = self.component_kind_by_id[:, np.clip(self.geometry.link_boundary_id, 0,
                                                  MAX_BOUNDARY_IDS - 1)]
        has_char = self.characteristic_stencil is not None
        return {
            "device": self.device, "storage": "sparse_active", "geometry": self.geometry.label,
            "boundary_label": self.boundary.label, "model": self.material.model, "nx": self.nx,
            "ny": self.ny, "nz": self.nz, "n_active": int(self.n_active),
            "n_cut_links": int(self.geometry.n_links), "steps": int(self.steps),
            "time": float(self.time), "dx": float(self.dx), "dt": float(self.dt),
            "lattice_speed": float(self.lattice_speed),
            "collision_omega": float(self.collision_omega),
            "boundary_reconstruction": self.boundary_reconstruction_name,
            "population_reconstruction": "dirichlet_bfl_neumann_characteristic" if has_char
            else "bfl",
            "boundary_stencil_radius": 3 if has_char else 1,
            "characteristic_cut_links": int(np.count_nonzero(np.any(ck == BC_NEUMANN, axis=0)))
            if has_char else 0,
            "bfl_cut_links": int(np.count_nonzero(np.any(ck == BC_DIRICHLET, axis=0)))
            if has_char else int(self.geometry.n_links),
            "normal_jacobian": self.normal_jacobian_name,
            "neumann_solver": self.neumann_solver_name,
            "has_neumann_cut_links": bool(self._has_neumann_cut_links),
            "surface_tangent_lsq_active": bool(self.tangent_lsq_active),
            "compatibility_projection": {"interval": 0, "active_in_step": False},
            "local_method": {
                "displacement_interval": int(self.local_displacement_interval),
                "displacement_sweeps": int(self.local_displacement_sweeps),
                "displacement_relax": float(self.local_displacement_relax),
                "boundary_weight": float(self.local_displacement_boundary_weight),
                "boundary_id": int(self.local_displacement_boundary_id),
                "F_repair_interval": int(self.local_compatibility_interval),
                "F_repair_blend": float(self.local_compatibility_blend),
                "kernel_stencil_radius": 2 if self.local_compatibility_interval > 0
                else (1 if drad > 0 else 0),
                "displacement_dependency_radius": drad,
                "composed_compatibility_radius": crad,
            },
            "memory_estimate_MiB": {k: float(v / 1024**2) for k, v in mem.items()},
            "max_abs_u": float(red["max_abs_u"]) if self.n_active else 0.0,
            "max_abs_v": float(red["max_abs_v"]) if self.n_active else 0.0,
            "min_J": float(red["min_J"]) if self.n_active else 0.0,
            "max_J": float(red["max_J"]) if self.n_active else 0.0,
            "finite": red["finite"] if self.n_active else False,
        }

    # -- exact checkpoint / restart (no counterpart in the reference) --------
    def _checkpoint_stamp(self) -> str:
        g = self.geometry
        cs = self.characteristic_stencil
        arrays = [self.active_i, self.active_j, self.active_k]
        arrays += [getattr(g, k) for k in ("link_i", "link_j", "link_k", "link_q",
                                            "link_boundary_id", "link_eta", "link_xb", "link_yb",
                                            "link_zb", "link_nx", "link_ny", "link_nz")]
        arrays += [None] if cs is None else [np.asarray(a) for a in cs]
        return _stamp.config_stamp(
            self, geometry_arrays=arrays,
            boundary_tables=(self.kind_by_id, self.mode_by_id, self.params_by_id))

    def checkpoint(self, path):
        """Write the complete stepping state (active populations, u*, U, u,
        time and step count) so that `restore` on a solver built with the
        same geometry and settings continues bit for bit.  (`save_npz` writes
        the reference's output format, which lacks u*.)"""
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        np.savez(path, f0=self._host(self.f0), u_star=self._host(self.u_star),
                 U=self._host(self.U), u=self._host(self.u), time=np.array(self.time),
                 steps=np.array(self.steps), stamp=np.array(self._checkpoint_stamp()))

    def restore(self, path):
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

    def save_npz(self, path):
        self.refresh_current()
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        xa, ya, za = self.active_coordinates()
        U = self.active_system_state()
        u = self.active_displacement()
        F = _state_to_F_np(U)
        P = _first_piola_np(F, self.material)
        J = np.maximum(_det3_np(F), self.jacobian_floor)
        sigma = np.einsum("ia...,ja...->ij...", P, F) / J
        np.savez_compressed(
            path, x_active=xa, y_active=ya, z_active=za, active_i=self.active_i,
            active_j=self.active_j, active_k=self.active_k,
            shape=np.array([self.nx, self.ny, self.nz], dtype=np.int32), dx=np.array(self.dx),
            dy=np.array(self.dy), dz=np.array(self.dz), u=u, U=U, F=F, P=P, sigma=sigma,
            time=np.array(self.time), storage=np.array("sparse_active"),
            metadata=np.array(json.dumps(self.summary())))


class _Graph3D:
    """Executable CUDA graph of ``nsteps`` (even) steps of one 3-D solver."""

    def __init__(self, solver: WarpSparseCurvedBoundaryLBM3D, nsteps: int) -> None:
        import ctypes

        if nsteps <= 0 or nsteps % 2:
            raise ValueError("graph step count must be a positive even number")
        self.solver, self.nsteps, self.step0 = solver, nsteps, solver.steps
        handle = ctypes.c_void_p()
        _native.check(solver._lib.cvlbm3d_graph_create(solver._problem, solver._fields(),
                                                       solver.steps, nsteps, ctypes.byref(handle)),
                      "cvlbm3d_graph_create")
        self.handle = handle

    def launch(self) -> None:
        s = self.solver
        for iv in (s.local_displacement_interval, s.local_compatibility_interval):
            if iv > 0 and (s.steps - self.step0) % iv != 0:
                raise RuntimeError("graph replay at a step phase different from its capture")
        s._clock.fill_(float(s.time))
        _native.check(s._lib.cvlbm_graph_launch(self.handle, s._stream()), "cvlbm_graph_launch")
        for _ in range(self.nsteps):
            s.time += s.dt
        s.steps += self.nsteps

    def __del__(self) -> None:
        try:
            if self.handle:
                self.solver._lib.cvlbm_graph_destroy(self.handle)
        except Exception:
            pass


WarpCurvedBoundaryLBM3D = WarpSparseCurvedBoundaryLBM3D


def relative_l2_active(error, reference, mask):
    e, r = np.asarray(error), np.asarray(reference)
    m = np.asarray(mask, dtype=bool)
    num = float(np.sqrt(np.sum(e[..., m] ** 2)))
    den = float(np.sqrt(np.sum(r[..., m] ** 2)))
    return num / max(den, np.finfo(float).eps)
