"""Host-side 3-D curved-boundary geometry and sparse connectivity.

Restates the reference's preprocessing in
``src/curved_lbm/three_d/curved_boundary_warp3d.py``: level-set cut links
(:332-721, both the per-point and the vectorised path, which order links
differently), the sphere and spherical-shell helpers (:723-800), the
active-node compaction and 6-neighbour table (:3683-3722) and the
surface-tangent LSQ weights of compat_bfl (:3725-3849).  Tables equal the
reference's element for element (fixtures ``tests/golden/g3_*`` and
``geo3_*`` pin this).
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, Literal

import numpy as np

from .vector_nonlinear_elastic_warp3d import BC_DIRICHLET, BC_NEUMANN, _cofactor_np, _first_piola_np

DIRS3 = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1]],
                 dtype=np.int32)
MAX_LSQ_STENCIL = 32
MAX_BOUNDARY_IDS = 16
BOUNDARY_ID_OUTER = 1
BOUNDARY_ID_INNER = 2

BoundaryKind = Literal["dirichlet", "neumann"]


def _kind_id(k: str) -> int:
    if k == "dirichlet":
        return BC_DIRICHLET
    if k == "neumann":
        return BC_NEUMANN
    raise ValueError(k)


@dataclass(frozen=True)
class CurvedBoundarySpec3D:
    """Boundary data per boundary id and displacement component (reference :194-258)."""

    kind: BoundaryKind = "dirichlet"
    value_mode: int = 0
    params: tuple[float, ...] = ()
    id_kinds: dict | None = None
    id_value_modes: dict | None = None
    id_params: dict | None = None
    label: str = ""
    component_kinds: tuple | None = None
    id_component_kinds: dict | None = None

    def tables(self, max_ids: int = MAX_BOUNDARY_IDS):
        kind = np.full(max_ids, _kind_id(self.kind), dtype=np.int32)
        mode = np.full(max_ids, int(self.value_mode), dtype=np.int32)
        p0 = np.zeros(16, dtype=np.float64)
        for i, v in enumerate(tuple(self.params)[:16]):
            p0[i] = float(v)
        params = np.tile(p0[None, :], (max_ids, 1))
        for i, v in (self.id_kinds or {}).items():
            if 0 <= int(i) < max_ids:
                kind[int(i)] = _kind_id(v)
        for i, v in (self.id_value_modes or {}).items():
            if 0 <= int(i) < max_ids:
                mode[int(i)] = int(v)
        for i, vals in (self.id_params or {}).items():
            if 0 <= int(i) < max_ids:
                params[int(i), :] = 0.0
                for j, v in enumerate(tuple(vals)[:16]):
                    params[int(i), j] = float(v)
        return kind, mode, np.ascontiguousarray(params)

    def component_kind_table(self, max_ids: int = MAX_BOUNDARY_IDS) -> np.ndarray:
        kind, _, _ = self.tables(max_ids)
        out = np.repeat(kind[None, :], 3, axis=0)
        if self.component_kinds is not None:
            vals = tuple(self.component_kinds)
            if len(vals) != 3:
                raise ValueError("component_kinds must contain exactly three kinds")
            for comp, v in enumerate(vals):
                out[comp, :] = _kind_id(v)
            for i, v in (self.id_kinds or {}).items():
                if 0 <= int(i) < max_ids:
                    out[:, int(i)] = _kind_id(v)
        for i, vals in (self.id_component_kinds or {}).items():
            if not 0 <= int(i) < max_ids:
                continue
            cv = tuple(vals)
            if len(cv) != 3:
                raise ValueError("id_component_kinds values must contain exactly three kinds")
            for comp, v in enumerate(cv):
                out[comp, int(i)] = _kind_id(v)
        return np.ascontiguousarray(out)


@dataclass(frozen=True)
class SphereDomain:
    center: tuple = (0.5, 0.5, 0.5)
    radius: float = 0.35

    def phi(self, x, y, z):
        cx, cy, cz = self.center
        return math.sqrt((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) - self.radius

    def normal(self, x, y, z):
        cx, cy, cz = self.center
        rx, ry, rz = x - cx, y - cy, z - cz
        r = max(math.sqrt(rx * rx + ry * ry + rz * rz), 1e-30)
        return rx / r, ry / r, rz / r


@dataclass
class CurvedBoundaryGeometry3D:
    nx: int
    ny: int
    nz: int
    length_x: float
    length_y: float
    length_z: float
    active: np.ndarray
    link_i: np.ndarray
    link_j: np.ndarray
    link_k: np.ndarray
    link_q: np.ndarray
    link_boundary_id: np.ndarray
    link_eta: np.ndarray
    link_xb: np.ndarray
    link_yb: np.ndarray
    link_zb: np.ndarray
    link_nx: np.ndarray
    link_ny: np.ndarray
    link_nz: np.ndarray
    label: str = "implicit"

    @property
    def dx(self):
        return self.length_x / float(self.nx)

    @property
    def dy(self):
        return self.length_y / float(self.ny)

    @property
    def dz(self):
        return self.length_z / float(self.nz)

    @property
    def n_active(self):
        return int(np.count_nonzero(self.active))

    @property
    def n_links(self):
        return int(self.link_i.size)

    def as_metadata(self):
        return {"label": self.label, "nx": self.nx, "ny": self.ny, "nz": self.nz,
                "dx": self.dx, "dy": self.dy, "dz": self.dz, "n_active": self.n_active,
                "n_cut_links": self.n_links}

    @classmethod
    def from_level_set(cls, *, nx: int, ny: int, nz: int, length_x: float, length_y: float,
                       length_z: float, phi: Callable, normal: Callable | None = None,
                       boundary_id: Callable | None = None, label: str = "level_set",
                       root_iterations: int = 42, phi_vectorized: Callable | None = None,
                       normal_vectorized: Callable | None = None, phi_chunk_size: int = 64):
        """Material where phi <= 0; links by bisection (reference :332-721)."""
        dx, dy, dz = length_x / nx, length_y / ny, length_z / nz
        if nx < 4 or ny < 4 or nz < 4:
            raise ValueError("nx,ny,nz>=4 required")
        if max(abs(dx - dy), abs(dx - dz)) > 1e-14:
            raise ValueError("D3Q6 requires dx=dy=dz")
        xs = (np.arange(nx) + 0.5) * dx
        ys = (np.arange(ny) + 0.5) * dy
        zs = (np.arange(nz) + 0.5) * dz
        ph = np.empty((nx, ny, nz), float)
        if phi_vectorized is None:
            for i, x in enumerate(xs):
                for j, y in enumerate(ys):
                    for k, z in enumerate(zs):
                        ph[i, j, k] = float(phi(float(x), float(y), float(z)))
        else:
            X2, Y2 = np.meshgrid(xs, ys, indexing="ij")
            chunk = max(1, int(phi_chunk_size))
            for k0 in range(0, nz, chunk):
                k1 = min(nz, k0 + chunk)
                vals = np.asarray(phi_vectorized(X2[:, :, None], Y2[:, :, None],
                                                 zs[None, None, k0:k1]), dtype=float)
                if vals.shape != ph[:, :, k0:k1].shape:
                    vals = np.broadcast_to(vals, ph[:, :, k0:k1].shape)
                ph[:, :, k0:k1] = vals
        active = ph <= 0.0
        if not np.any(active):
            raise ValueError("no active material nodes")

        def unit_normal(a, b, c):
            r = max(math.sqrt(a * a + b * b + c * c), 1.0e-30)
            return a / r, b / r, c / r

        def point_normal(x, y, z):
            if normal is not None:
                a, b, c = normal(float(x), float(y), float(z))
                return unit_normal(float(a), float(b), float(c))
            h = 0.5 * dx
            a = (float(phi(float(x) + h, float(y), float(z)))
                 - float(phi(float(x) - h, float(y), float(z)))) / (2 * h)
            b = (float(phi(float(x), float(y) + h, float(z)))
                 - float(phi(float(x), float(y) - h, float(z)))) / (2 * h)
            c = (float(phi(float(x), float(y), float(z) + h))
                 - float(phi(float(x), float(y), float(z) - h))) / (2 * h)
            return unit_normal(a, b, c)

        def clamp_bid(b):
            return max(0, min(MAX_BOUNDARY_IDS - 1, int(b)))

        sample = np.linspace(0.0, 1.0, 17)
        if phi_vectorized is not None:
            return cls._vectorized_links(
                nx, ny, nz, length_x, length_y, length_z, dx, dy, dz, xs, ys, zs, ph, active,
                phi_vectorized, normal_vectorized, point_normal, boundary_id, root_iterations,
                sample, label)
        rows = []

        def phis(x, y, z):
            return float(phi(float(x), float(y), float(z)))

        for i, x0 in enumerate(xs):
            for j, y0 in enumerate(ys):
                for k, z0 in enumerate(zs):
                    if not active[i, j, k]:
                        continue
                    p0 = ph[i, j, k]
                    for q, (di, dj, dk) in enumerate(DIRS3):
                        ii, jj, kk = i + int(di), j + int(dj), k + int(dk)
                        if 0 <= ii < nx and 0 <= jj < ny and 0 <= kk < nz and active[ii, jj, kk]:
                            continue
                        x1, y1, z1 = x0 + di * dx, y0 + dj * dy, z0 + dk * dz
                        p1 = phis(x1, y1, z1)
                        if p0 <= 0 and p1 >= 0:
                            lo, hi = 0.0, 1.0
                        else:
                            vals = [phis(x0 + s * (x1 - x0), y0 + s * (y1 - y0), z0 + s * (z1 - z0))
                                    for s in sample]
                            idx = next((m for m in range(len(sample) - 1)
                                        if vals[m] <= 0 and vals[m + 1] >= 0), None)
                            lo, hi = ((0.5, 0.5) if idx is None
                                      else (float(sample[idx]), float(sample[idx + 1])))
                        for _ in range(root_iterations):
                            mid = 0.5 * (lo + hi)
                            if phis(x0 + mid * (x1 - x0), y0 + mid * (y1 - y0),
                                    z0 + mid * (z1 - z0)) <= 0:
                                lo = mid
                            else:
                                hi = mid
                        eta = float(np.clip(0.5 * (lo + hi), 1e-6, 1 - 1e-6))
                        xb, yb, zb = x0 + eta * (x1 - x0), y0 + eta * (y1 - y0), z0 + eta * (z1 - z0)
                        nxv, nyv, nzv = point_normal(xb, yb, zb)
                        bid = 1 if boundary_id is None else int(boundary_id(xb, yb, zb, nxv, nyv, nzv))
                        rows.append((i, j, k, q, clamp_bid(bid), eta, xb, yb, zb, nxv, nyv, nzv))
        cols = list(zip(*rows)) if rows else [()] * 12
        ints = [np.ascontiguousarray(np.array(c, np.int32)) for c in cols[:5]]
        reals = [np.ascontiguousarray(np.array(c, float)) for c in cols[5:]]
        return cls(nx, ny, nz, float(length_x), float(length_y), float(length_z),
                   np.ascontiguousarray(active.astype(np.int32)), *ints, *reals, label)

    @classmethod
    def _vectorized_links(cls, nx, ny, nz, length_x, length_y, length_z, dx, dy, dz, xs, ys, zs,
                          ph, active, phi_vectorized, normal_vectorized, point_normal,
                          boundary_id, root_iterations, sample, label):
        def phiv(x, y, z):
            out = np.asarray(phi_vectorized(np.asarray(x), np.asarray(y), np.asarray(z)),
                             dtype=float)
            shape = np.broadcast(x, y, z).shape
            return out if out.shape == shape else np.broadcast_to(out, shape)

        def normalv(x, y, z):
            shape = np.broadcast(x, y, z).shape
            if normal_vectorized is not None:
                vals = normal_vectorized(np.asarray(x), np.asarray(y), np.asarray(z))
                if isinstance(vals, (tuple, list)):
                    a, b, c = (np.asarray(v, dtype=float) for v in vals[:3])
                else:
                    arr = np.asarray(vals, dtype=float)
                    if arr.shape[:1] == (3,):
                        a, b, c = arr[0], arr[1], arr[2]
                    elif arr.shape[-1:] == (3,):
                        a, b, c = arr[..., 0], arr[..., 1], arr[..., 2]
                    else:
                        raise ValueError(
                            "normal_vectorized must return a 3-tuple or an array with a 3-vector axis")
                a = np.broadcast_to(a, shape).astype(float, copy=False)
                b = np.broadcast_to(b, shape).astype(float, copy=False)
                c = np.broadcast_to(c, shape).astype(float, copy=False)
                r = np.maximum(np.sqrt(a * a + b * b + c * c), 1.0e-30)
                return a / r, b / r, c / r
            a = np.empty(shape)
            b = np.empty(shape)
            c = np.empty(shape)
            flat = [np.broadcast_to(v, shape).reshape(-1) for v in (x, y, z)]
            for m in range(a.size):
                a.flat[m], b.flat[m], c.flat[m] = point_normal(flat[0][m], flat[1][m], flat[2][m])
            return a, b, c

        parts = []
        for q, (di, dj, dk) in enumerate(DIRS3):
            nb = np.zeros_like(active, dtype=bool)
            if di == 1:
                nb[:-1, :, :] = active[1:, :, :]
            elif di == -1:
                nb[1:, :, :] = active[:-1, :, :]
            elif dj == 1:
                nb[:, :-1, :] = active[:, 1:, :]
            elif dj == -1:
                nb[:, 1:, :] = active[:, :-1, :]
            elif dk == 1:
                nb[:, :, :-1] = active[:, :, 1:]
            elif dk == -1:
                nb[:, :, 1:] = active[:, :, :-1]
            ii, jj, kk = np.nonzero(active & ~nb)
            if ii.size == 0:
                continue
            x0, y0, z0 = xs[ii], ys[jj], zs[kk]
            x1, y1, z1 = x0 + float(di) * dx, y0 + float(dj) * dy, z0 + float(dk) * dz
            p0 = ph[ii, jj, kk]
            p1 = phiv(x1, y1, z1)
            lo = np.zeros(ii.size)
            hi = np.ones(ii.size)
            needs = np.where(~((p0 <= 0.0) & (p1 >= 0.0)))[0]
            if needs.size:
                found = np.zeros(needs.size, dtype=bool)
                lo_n = np.full(needs.size, 0.5)
                hi_n = np.full(needs.size, 0.5)
                prev_s, prev_v = sample[0], p0[needs]
                for ss in sample[1:]:
                    pm = phiv(x0[needs] + ss * (x1[needs] - x0[needs]),
                              y0[needs] + ss * (y1[needs] - y0[needs]),
                              z0[needs] + ss * (z1[needs] - z0[needs]))
                    hit = (~found) & (prev_v <= 0.0) & (pm >= 0.0)
                    lo_n[hit] = prev_s
                    hi_n[hit] = ss
                    found[hit] = True
                    prev_s, prev_v = ss, pm
                lo[needs] = lo_n
                hi[needs] = hi_n
            for _ in range(root_iterations):
                mid = 0.5 * (lo + hi)
                inside = phiv(x0 + mid * (x1 - x0), y0 + mid * (y1 - y0), z0 + mid * (z1 - z0)) <= 0.0
                lo = np.where(inside, mid, lo)
                hi = np.where(inside, hi, mid)
            eta = np.clip(0.5 * (lo + hi), 1.0e-6, 1.0 - 1.0e-6)
            xb, yb, zb = x0 + eta * (x1 - x0), y0 + eta * (y1 - y0), z0 + eta * (z1 - z0)
            nxv, nyv, nzv = normalv(xb, yb, zb)
            if boundary_id is None:
                bid = np.ones(ii.size, dtype=np.int32)
            else:
                bid = np.array([int(boundary_id(float(xb[m]), float(yb[m]), float(zb[m]),
                                                float(nxv[m]), float(nyv[m]), float(nzv[m])))
                                for m in range(ii.size)], dtype=np.int32)
            parts.append((ii.astype(np.int32), jj.astype(np.int32), kk.astype(np.int32),
                          np.full(ii.size, q, dtype=np.int32),
                          np.clip(bid, 0, MAX_BOUNDARY_IDS - 1).astype(np.int32), eta, xb, yb, zb,
                          np.asarray(nxv, float), np.asarray(nyv, float), np.asarray(nzv, float)))

        def cat(idx, dtype):
            if parts:
                return np.ascontiguousarray(np.concatenate([p[idx] for p in parts]).astype(dtype, copy=False))
            return np.ascontiguousarray(np.empty(0, dtype=dtype))

        cols = [cat(k, np.int32) for k in range(5)] + [cat(k, float) for k in range(5, 12)]
        return cls(nx, ny, nz, float(length_x), float(length_y), float(length_z),
                   np.ascontiguousarray(active.astype(np.int32)), *cols, label)

    @classmethod
    def sphere(cls, *, nx, ny, nz, length_x=1.0, length_y=1.0, length_z=1.0,
               center=(0.5, 0.5, 0.5), radius=0.35):
        sph = SphereDomain(center, radius)
        return cls.from_level_set(nx=nx, ny=ny, nz=nz, length_x=length_x, length_y=length_y,
                                  length_z=length_z, phi=sph.phi, normal=sph.normal,
                                  label=f"sphere(center={center},r={radius})")

    @classmethod
    def spherical_shell(cls, *, nx, ny, nz, length_x=1.0, length_y=1.0, length_z=1.0,
                        center=(0.5, 0.5, 0.5), inner_radius=0.18, outer_radius=0.42):
        if not (0.0 < inner_radius < outer_radius):
            raise ValueError("spherical_shell requires 0 < inner_radius < outer_radius")
        cx, cy, cz = center

        def rr(x, y, z):
            return math.sqrt((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2)

        def inner(r):
            return abs(r - inner_radius) <= abs(r - outer_radius)

        def phi(x, y, z):
            r = rr(x, y, z)
            return max(r - outer_radius, inner_radius - r)

        def normal(x, y, z):
            r = max(rr(x, y, z), 1.0e-30)
            ex, ey, ez = (x - cx) / r, (y - cy) / r, (z - cz) / r
            return (-ex, -ey, -ez) if inner(r) else (ex, ey, ez)

        def bid(x, y, z, _a, _b, _c):
            return BOUNDARY_ID_INNER if inner(rr(x, y, z)) else BOUNDARY_ID_OUTER

        return cls.from_level_set(
            nx=nx, ny=ny, nz=nz, length_x=length_x, length_y=length_y, length_z=length_z,
            phi=phi, normal=normal, boundary_id=bid,
            label=f"spherical_shell(center={center},ri={inner_radius},ro={outer_radius})")


def _sparse_tables_from_geometry(geometry: CurvedBoundaryGeometry3D) -> dict:
    """Active-node ids, 6-neighbour table and link node/upstream ids (reference :3683-3722)."""
    act = np.asarray(geometry.active, dtype=bool)
    ai, aj, ak = (np.ascontiguousarray(a.astype(np.int32)) for a in np.nonzero(act))
    n = int(ai.size)
    active_id = np.full(act.shape, -1, dtype=np.int32)
    active_id[ai, aj, ak] = np.arange(n, dtype=np.int32)
    nx, ny, nz = geometry.nx, geometry.ny, geometry.nz
    neighbor = np.full((6, n), -1, dtype=np.int32)
    for q, (di, dj, dk) in enumerate(DIRS3):
        ii, jj, kk = ai + int(di), aj + int(dj), ak + int(dk)
        ok = (ii >= 0) & (ii < nx) & (jj >= 0) & (jj < ny) & (kk >= 0) & (kk < nz)
        v = np.where(ok)[0]
        if v.size:
            neighbor[q, v] = active_id[ii[v], jj[v], kk[v]]
    li, lj, lk = geometry.link_i, geometry.link_j, geometry.link_k
    link_p = active_id[li, lj, lk].astype(np.int32)
    up = np.full(geometry.n_links, -1, dtype=np.int32)
    if geometry.n_links:
        d = DIRS3[np.asarray(geometry.link_q)]
        ui, uj, uk = li - d[:, 0], lj - d[:, 1], lk - d[:, 2]
        ok = (ui >= 0) & (ui < nx) & (uj >= 0) & (uj < ny) & (uk >= 0) & (uk < nz)
        up[ok] = active_id[ui[ok], uj[ok], uk[ok]]
    return {"active_i": ai, "active_j": aj, "active_k": ak,
            "active_id": np.ascontiguousarray(active_id), "neighbor": np.ascontiguousarray(neighbor),
            "link_p": np.ascontiguousarray(link_p), "link_upstream": np.ascontiguousarray(up)}


def _basis_np(n):
    """Tangent pair of a normal (reference :886-892)."""
    n = np.asarray(n, float)
    n = n / max(np.linalg.norm(n), np.finfo(float).eps)
    ref = np.array([1.0, 0, 0]) if abs(n[0]) < 0.75 else np.array([0, 1.0, 0])
    t1 = np.cross(n, ref)
    t1 = t1 / max(np.linalg.norm(t1), np.finfo(float).eps)
    return t1, np.cross(n, t1)


def _build_sparse_tangent_lsq_weights(geometry, tables, *, max_stencil: int = MAX_LSQ_STENCIL):
    """Two surface-tangent derivative stencils per link for compat_bfl (reference :3725-3849)."""
    n_links = int(geometry.n_links)
    out_p = np.full((n_links, max_stencil), -1, dtype=np.int32)
    wt1 = np.zeros((n_links, max_stencil))
    wt2 = np.zeros((n_links, max_stencil))
    valid = np.zeros(n_links, dtype=np.int32)
    if n_links == 0:
        return {"lsq_p": out_p, "lsq_wt1": wt1, "lsq_wt2": wt2, "lsq_valid": valid}
    act = np.asarray(geometry.active, dtype=bool)
    active_id = np.asarray(tables["active_id"], dtype=np.int32)
    nx, ny, nz = geometry.nx, geometry.ny, geometry.nz
    dx, dy, dz = float(geometry.dx), float(geometry.dy), float(geometry.dz)
    xs = (np.arange(nx, dtype=np.float64) + 0.5) * dx
    ys = (np.arange(ny, dtype=np.float64) + 0.5) * dy
    zs = (np.arange(nz, dtype=np.float64) + 0.5) * dz
    eye10 = np.eye(10, dtype=np.float64)

    def fit(ell, radius):
        xb, yb, zb = (float(geometry.link_xb[ell]), float(geometry.link_yb[ell]),
                      float(geometry.link_zb[ell]))
        nvec = np.array([geometry.link_nx[ell], geometry.link_ny[ell], geometry.link_nz[ell]],
                        dtype=np.float64)
        nvec = nvec / max(float(np.linalg.norm(nvec)), np.finfo(float).eps)
        t1, t2 = _basis_np(nvec)
        i0, j0, k0 = int(geometry.link_i[ell]), int(geometry.link_j[ell]), int(geometry.link_k[ell])
        cand = []
        r2max = (float(radius) + 0.25) ** 2
        for ii in range(max(0, i0 - radius), min(nx, i0 + radius + 1)):
            for jj in range(max(0, j0 - radius), min(ny, j0 + radius + 1)):
                for kk in range(max(0, k0 - radius), min(nz, k0 + radius + 1)):
                    if not act[ii, jj, kk]:
                        continue
                    p = int(active_id[ii, jj, kk])
                    if p < 0:
                        continue
                    rx, ry, rz = (float(xs[ii]) - xb) / dx, (float(ys[jj]) - yb) / dy, (float(zs[kk]) - zb) / dz
                    r2 = rx * rx + ry * ry + rz * rz
                    if r2 <= r2max:
                        cand.append((r2, p, rx, ry, rz))
        cand.sort(key=lambda it: it[0])
        if len(cand) < 10:
            return None
        cand = cand[:max_stencil]
        k = len(cand)
        A = np.empty((k, 10))
        wd = np.empty(k)
        for m, (r2, _p, rx, ry, rz) in enumerate(cand):
            A[m] = (1.0, rx, ry, rz, 0.5 * rx * rx, rx * ry, rx * rz, 0.5 * ry * ry, ry * rz,
                    0.5 * rz * rz)
            wd[m] = math.exp(-0.5 * r2 / (1.75 * 1.75)) + 1.0e-4
        if np.linalg.matrix_rank(A, tol=1.0e-10) < 10:
            return None
        M = A.T @ (A * wd[:, None])
        cond = np.linalg.cond(M)
        if not np.isfinite(cond) or cond > 1.0e9:
            return None
        try:
            c2v = np.linalg.solve(M + 1.0e-12 * eye10, A.T * wd[None, :])
        except np.linalg.LinAlgError:
            return None
        w1 = np.array([0.0, t1[0] / dx, t1[1] / dy, t1[2] / dz, 0, 0, 0, 0, 0, 0], dtype=np.float64) @ c2v
        w2 = np.array([0.0, t2[0] / dx, t2[1] / dy, t2[2] / dz, 0, 0, 0, 0, 0, 0], dtype=np.float64) @ c2v
        h = max(dx, dy, dz)
        if (not np.all(np.isfinite(w1))) or (not np.all(np.isfinite(w2))):
            return None
        if abs(float(np.sum(w1))) * h > 1.0e-6 or abs(float(np.sum(w2))) * h > 1.0e-6:
            return None
        if float(np.sum(np.abs(w1))) * h > 12.0 or float(np.sum(np.abs(w2))) * h > 12.0:
            return None
        return cand, w1, w2

    for ell in range(n_links):
        res = None
        for radius in (3, 4, 5):
            res = fit(ell, radius)
            if res is not None:
                break
        if res is None:
            continue
        cand, w1, w2 = res
        for m, (_r2, p, _x, _y, _z) in enumerate(cand):
            out_p[ell, m] = int(p)
            wt1[ell, m] = float(w1[m])
            wt2[ell, m] = float(w2[m])
        valid[ell] = 1
    return {"lsq_p": np.ascontiguousarray(out_p), "lsq_wt1": np.ascontiguousarray(wt1),
            "lsq_wt2": np.ascontiguousarray(wt2), "lsq_valid": np.ascontiguousarray(valid)}


def _affine_neo_hooke_F_P_np(p, t):
    pp = np.zeros(16)
    pp[: min(16, len(p))] = p[: min(16, len(p))]
    tt = float(t) if pp[11] <= 0.0 else min(float(t), float(pp[11]))
    F = np.eye(3) + tt * pp[:9].reshape(3, 3)
    J = float(np.linalg.det(F))
    H = _cofactor_np(F) / max(J, np.finfo(float).eps)
    lam, mu = float(pp[9]), float(pp[10])
    return F, mu * (F - H) + 0.5 * lam * (J * J - 1.0) * H


def _value_np(mode, p, comp, x, y, z, n, t):
    """Host boundary value (reference :818-883)."""
    pp = np.zeros(16)
    pp[: min(16, len(p))] = p[: min(16, len(p))]
    if mode == 0:
        return 0.0
    if mode == 1:
        return float(pp[comp])
    if mode == 200:
        scale = 1.0 if pp[3] <= 0 or t >= pp[3] else math.sin(math.pi * t / pp[3]) ** 2
        return float(pp[comp] * scale)
    if mode == 4:
        if pp[12] > 0 and t > pp[12]:
            return 0.0
        return float((pp[:9].reshape(3, 3) @ np.array([x, y, z]) + pp[9:12])[comp])
    if mode == 204:
        act = float(pp[3])
        den = float(pp[4]) if pp[4] > 0 else 2.0 * act
        scale = 1.0 if act <= 0 or t >= act else math.sin(math.pi * t / den) ** 2
        return float(pp[comp] * scale)
    if mode == 201:
        return float(pp[:9].reshape(3, 3)[comp, :] @ n)
    if mode == 205:
        _, P = _affine_neo_hooke_F_P_np(pp, t)
        return float(P[comp, :] @ n)
    if mode == 202:
        return float(pp[0] * n[comp])
    if mode == 203:
        act = float(pp[1])
        den = float(pp[2]) if pp[2] > 0 else 2.0 * act
        scale = 1.0 if act <= 0 or t >= act else math.sin(math.pi * t / den) ** 2
        return float(pp[0] * scale * n[comp])
    if mode == 208:
        scale = 1.0 if pp[1] <= 0 or t >= pp[1] else t / pp[1]
        return float(pp[0] * scale * n[comp])
    if mode == 206:
        act = float(pp[4])
        den = float(pp[5]) if pp[5] > 0 else 2.0 * act
        scale = 1.0 if act <= 0 or t >= act else math.sin(math.pi * t / den) ** 2
        ddx, ddy = x - float(pp[0]), y - float(pp[1])
        return float((-scale * pp[3] * ddy, scale * pp[3] * ddx, scale * pp[2])[comp])
    if mode == 207:
        act = float(pp[4])
        if act <= 0.0 or t >= act:
            return 0.0
        phase = math.pi * t / act
        s = 0.5 * (1.0 - math.cos(phase))
        sdot = 0.5 * math.pi / act * math.sin(phase)
        th, thd = float(pp[3]) * s, float(pp[3]) * sdot
        ddx, ddy = x - float(pp[0]), y - float(pp[1])
        vals = (thd * (-math.sin(th) * ddx - math.cos(th) * ddy),
                thd * (math.cos(th) * ddx - math.sin(th) * ddy), float(pp[2]) * sdot)
        return float(vals[comp])
    return 0.0


def _solve_Fb_np(Fg, n, T, mat, j_floor=1e-12):
    """Host Newton for P(F_b) n = T (reference :895-931)."""
    n = np.asarray(n, float)
    n = n / max(np.linalg.norm(n), np.finfo(float).eps)
    t1, t2 = _basis_np(n)
    Fg = np.asarray(Fg, float).reshape(3, 3)
    h = Fg @ n
    g1, g2 = Fg @ t1, Fg @ t2

    def make(hv):
        return np.outer(hv, n) + np.outer(g1, t1) + np.outer(g2, t2)

    def res(hv):
        return _first_piola_np(make(hv), mat) @ n - T

    for _ in range(24):
        r = res(h)
        if np.linalg.norm(r) < 1e-11:
            break
        Jm = np.zeros((3, 3))
        for a in range(3):
            hp = h.copy()
            hp[a] += 1e-6
            Jm[:, a] = (res(hp) - r) / 1e-6
        try:
            d = np.linalg.solve(Jm, -r)
        except np.linalg.LinAlgError:
            break
        step = 1.0
        for _ls in range(16):
            hc = h + step * d
            if np.linalg.det(make(hc)) > j_floor:
                h = hc
                break
            step *= 0.5
    return make(h)


def constant_piola_params3d(material, F):
    return tuple(float(x) for x in _first_piola_np(np.asarray(F, float).reshape(3, 3), material).reshape(-1))
