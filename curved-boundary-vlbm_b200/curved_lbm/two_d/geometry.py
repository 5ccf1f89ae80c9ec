"""Host-side 2-D curved-boundary geometry: level-set cut links and weights.

Restates the reference's geometry preprocessing
(``src/curved_lbm/two_d/curved_boundary_warp.py`` :332-932).  The tables it
produces are inputs of the time step, so they must equal the reference's
element for element: the same ``phi`` calls, the same bisection sequence and
the same NumPy linear algebra in the same order.  The fixture
``tests/golden/geo2_*.npz`` (generated by the reference itself) pins this.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable

import numpy as np

from .vector_nonlinear_elastic_warp import Q, _CX, _CY

MAX_LSQ_STENCIL = 24
MAX_BOUNDARY_IDS = 8
BOUNDARY_ID_OUTER = 1
BOUNDARY_ID_INNER = 2

_PROBE_PAIRS = ((0.75, 1.75), (1.0, 2.0), (1.25, 2.5), (1.5, 3.0))
_SINGLE_PROBES = (0.75, 1.0, 1.25, 1.5, 2.0)


def _local_quadratic_fit(active, x_coords, y_coords, i0, j0, xb, yb, dx, max_stencil):
    """Weighted quadratic LSQ map from <=24 samples to polynomial coefficients.

    Samples are active nodes within a radius of three cells (r^2 <= 9.5 in
    cell units) of the cut point, nearest first.  Returns the candidate list
    and ``coeff_to_values`` (6 x k) or None when the fit is rank deficient or
    ill conditioned (reference :395-426 and :450-481, which build the same fit
    twice).
    """
    nx, ny = active.shape
    cand = []
    for ii in range(max(0, i0 - 3), min(nx, i0 + 4)):
        for jj in range(max(0, j0 - 3), min(ny, j0 + 4)):
            if active[ii, jj] == 0:
                continue
            rx = (float(x_coords[ii]) - xb) / dx
            ry = (float(y_coords[jj]) - yb) / dx
            r2 = rx * rx + ry * ry
            if r2 <= 9.5:
                cand.append((r2, ii, jj, rx, ry))
    cand.sort(key=lambda item: item[0])
    if len(cand) < 6:
        return None
    cand = cand[:max_stencil]
    k = len(cand)
    A = np.empty((k, 6), dtype=np.float64)
    wd = np.empty(k, dtype=np.float64)
    for m, (r2, _ii, _jj, rx, ry) in enumerate(cand):
        A[m] = (1.0, rx, ry, 0.5 * rx * rx, rx * ry, 0.5 * ry * ry)
        wd[m] = math.exp(-0.5 * r2 / (1.5 * 1.5)) + 1.0e-4
    if np.linalg.matrix_rank(A, tol=1.0e-10) < 6:
        return None
    M = A.T @ (A * wd[:, None])
    cond = np.linalg.cond(M)
    if not np.isfinite(cond) or cond > 1.0e8:
        return None
    try:
        c2v = np.linalg.solve(M + 1.0e-12 * np.eye(6, dtype=np.float64), A.T * wd[None, :])
    except np.linalg.LinAlgError:
        return None
    return cand, c2v


def _merge_slots(out_i, out_j, ell, cand, max_stencil):
    """Slot of every candidate, appending nodes not yet in the link's stencil."""
    slot_of = {}
    for m in range(max_stencil):
        if out_i[ell, m] >= 0 and out_j[ell, m] >= 0:
            slot_of[(int(out_i[ell, m]), int(out_j[ell, m]))] = m
    next_slot = len(slot_of)
    slots = []
    for _r2, ii, jj, _rx, _ry in cand:
        key = (int(ii), int(jj))
        s = slot_of.get(key)
        if s is None:
            if next_slot >= max_stencil:
                return None
            s = next_slot
            next_slot += 1
            slot_of[key] = s
            out_i[ell, s] = int(ii)
            out_j[ell, s] = int(jj)
        slots.append(s)
    return slots


def build_boundary_lsq_weights(*, active, x_coords, y_coords, link_i, link_j, link_xb, link_yb,
                               link_nx, link_ny, dx, max_stencil=MAX_LSQ_STENCIL):
    """Normal-probe value weights and tangent/gradient weights per cut link.

    Value: two probes X1 = Xb - h1 n, X2 = Xb - h2 n, bilinear interpolation,
    linear extrapolation back to Xb (first probe pair whose bilinear support is
    active), else one probe.  Tangent derivative and gradient: weighted
    quadratic LSQ.  Reference :332-606 (_build_boundary_lsq_weights).
    """
    n_links = int(link_i.size)
    nx, ny = active.shape
    out_i = np.full((n_links, max_stencil), -1, dtype=np.int32)
    out_j = np.full((n_links, max_stencil), -1, dtype=np.int32)
    out_w = np.zeros((n_links, max_stencil), dtype=np.float64)
    out_wt = np.zeros((n_links, max_stencil), dtype=np.float64)
    out_wx = np.zeros((n_links, max_stencil), dtype=np.float64)
    out_wy = np.zeros((n_links, max_stencil), dtype=np.float64)
    valid = np.zeros(n_links, dtype=np.int32)
    dx = float(dx)
    x0g = float(x_coords[0]) if len(x_coords) else 0.5 * dx
    y0g = float(y_coords[0]) if len(y_coords) else 0.5 * dx

    def bilinear(xp, yp):
        rx = (xp - x0g) / dx
        ry = (yp - y0g) / dx
        i0 = math.floor(rx)
        j0 = math.floor(ry)
        sx = rx - i0
        sy = ry - j0
        if i0 < 0 or j0 < 0 or i0 + 1 >= nx or j0 + 1 >= ny:
            return None
        nodes = ((i0, j0, (1.0 - sx) * (1.0 - sy)), (i0 + 1, j0, sx * (1.0 - sy)),
                 (i0, j0 + 1, (1.0 - sx) * sy), (i0 + 1, j0 + 1, sx * sy))
        for ii, jj, _w in nodes:
            if active[ii, jj] == 0:
                return None
        return nodes

    for ell in range(n_links):
        xb, yb = float(link_xb[ell]), float(link_yb[ell])
        nxb, nyb = float(link_nx[ell]), float(link_ny[ell])
        li, lj = int(link_i[ell]), int(link_j[ell])
        accum: dict = {}
        found = False
        for h1, h2 in _PROBE_PAIRS:
            w1 = bilinear(xb - h1 * dx * nxb, yb - h1 * dx * nyb)
            w2 = bilinear(xb - h2 * dx * nxb, yb - h2 * dx * nyb)
            if w1 is None or w2 is None:
                continue
            accum.clear()
            c1 = h2 / (h2 - h1)
            c2 = -h1 / (h2 - h1)
            for ii, jj, ww in w1:
                accum[(int(ii), int(jj))] = accum.get((int(ii), int(jj)), 0.0) + c1 * float(ww)
            for ii, jj, ww in w2:
                accum[(int(ii), int(jj))] = accum.get((int(ii), int(jj)), 0.0) + c2 * float(ww)
            found = True
            break
        if not found:
            for h in _SINGLE_PROBES:
                w1 = bilinear(xb - h * dx * nxb, yb - h * dx * nyb)
                if w1 is None:
                    continue
                accum.clear()
                for ii, jj, ww in w1:
                    accum[(int(ii), int(jj))] = accum.get((int(ii), int(jj)), 0.0) + float(ww)
                found = True
                break
        if not found:
            continue
        items = [(ij, w) for ij, w in accum.items() if abs(w) > 1.0e-14]
        items.sort(key=lambda it: (it[0][0] - li) ** 2 + (it[0][1] - lj) ** 2)
        if len(items) > max_stencil:
            continue
        if (not items or not np.isfinite([w for _ij, w in items]).all()
                or sum(abs(w) for _ij, w in items) > 3.5):
            continue
        for m, ((ii, jj), ww) in enumerate(items):
            out_i[ell, m] = int(ii)
            out_j[ell, m] = int(jj)
            out_w[ell, m] = float(ww)
        fit = _local_quadratic_fit(active, x_coords, y_coords, li, lj, xb, yb, dx, max_stencil)
        if fit is not None:
            cand, c2v = fit
            target = np.array([0.0, -nyb / dx, nxb / dx, 0.0, 0.0, 0.0], dtype=np.float64)
            wt = target @ c2v
            if (np.all(np.isfinite(wt)) and not abs(np.sum(wt)) * dx > 1.0e-6
                    and not np.sum(np.abs(wt)) * dx > 8.0):
                slots = _merge_slots(out_i, out_j, ell, cand, max_stencil)
                if slots is None:
                    out_wt[ell, :] = 0.0
                else:
                    for m, s in enumerate(slots):
                        out_wt[ell, s] = float(wt[m])
        if fit is not None:
            cand, c2v = fit
            wx = np.array([0.0, 1.0 / dx, 0.0, 0.0, 0.0, 0.0], dtype=np.float64) @ c2v
            wy = np.array([0.0, 0.0, 1.0 / dx, 0.0, 0.0, 0.0], dtype=np.float64) @ c2v
            if (np.all(np.isfinite(wx)) and np.all(np.isfinite(wy))
                    and not abs(np.sum(wx)) * dx > 1.0e-6 and not abs(np.sum(wy)) * dx > 1.0e-6
                    and not np.sum(np.abs(wx)) * dx > 12.0
                    and not np.sum(np.abs(wy)) * dx > 12.0):
                slots = _merge_slots(out_i, out_j, ell, cand, max_stencil)
                if slots is None:
                    out_wx[ell, :] = 0.0
                    out_wy[ell, :] = 0.0
                else:
                    for m, s in enumerate(slots):
                        out_wx[ell, s] = float(wx[m])
                        out_wy[ell, s] = float(wy[m])
        valid[ell] = 1
    return tuple(np.ascontiguousarray(a) for a in (out_i, out_j, out_w, out_wt, out_wx, out_wy,
                                                   valid))


@dataclass(frozen=True)
class CircleDomain:
    """Circle level set (reference :270-329)."""

    center_x: float = 0.5
    center_y: float = 0.5
    radius: float = 0.38

    def phi(self, x, y):
        return (np.sqrt((np.asarray(x) - self.center_x) ** 2 + (np.asarray(y) - self.center_y) ** 2)
                - self.radius)

    def normal(self, x, y):
        rx = np.asarray(x) - self.center_x
        ry = np.asarray(y) - self.center_y
        r = np.maximum(np.sqrt(rx * rx + ry * ry), np.finfo(float).eps)
        return rx / r, ry / r


def _bisect(phi, x0, y0, x1, y1, lo, hi, iterations):
    for _ in range(iterations):
        mid = 0.5 * (lo + hi)
        if phi(x0 + mid * (x1 - x0), y0 + mid * (y1 - y0)) <= 0.0:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


@dataclass
class CurvedBoundaryGeometry:
    """Active mask and cut-link data of an implicit 2-D domain (reference :609-932)."""

    nx: int
    ny: int
    length_x: float
    length_y: float
    active: np.ndarray
    link_i: np.ndarray
    link_j: np.ndarray
    link_q: np.ndarray
    link_boundary_id: np.ndarray
    link_eta: np.ndarray
    link_xb: np.ndarray
    link_yb: np.ndarray
    link_nx: np.ndarray
    link_ny: np.ndarray
    label: str = "implicit"
    lsq_i: np.ndarray | None = None
    lsq_j: np.ndarray | None = None
    lsq_wb: np.ndarray | None = None
    lsq_wt: np.ndarray | None = None
    lsq_wx: np.ndarray | None = None
    lsq_wy: np.ndarray | None = None
    lsq_valid: np.ndarray | None = None

    @property
    def dx(self) -> float:
        return self.length_x / float(self.nx)

    @property
    def dy(self) -> float:
        return self.length_y / float(self.ny)

    @property
    def n_active(self) -> int:
        return int(np.count_nonzero(self.active))

    @property
    def n_links(self) -> int:
        return int(self.link_i.size)

    def as_metadata(self) -> dict:
        return {
            "label": self.label, "nx": self.nx, "ny": self.ny, "length_x": self.length_x,
            "length_y": self.length_y, "dx": self.dx, "dy": self.dy, "n_active": self.n_active,
            "n_cut_links": self.n_links,
            "boundary_ids": sorted(int(v) for v in np.unique(self.link_boundary_id))
            if self.n_links else [],
        }

    @classmethod
    def from_level_set(cls, *, nx: int, ny: int, length_x: float, length_y: float,
                       phi: Callable[[float, float], float],
                       normal: Callable[[float, float], tuple[float, float]] | None = None,
                       boundary_id: Callable[[float, float, float, float], int] | None = None,
                       label: str = "level_set", root_iterations: int = 40
                       ) -> "CurvedBoundaryGeometry":
        """Material where phi <= 0; cut fractions by bisection (reference :668-858)."""
        if nx < 4 or ny < 4:
            raise ValueError("nx and ny must be at least four")
        dx = float(length_x) / float(nx)
        dy = float(length_y) / float(ny)
        if abs(dx - dy) > 1.0e-14:
            raise ValueError("D2Q4 curved-boundary implementation requires dx=dy")
        x = (np.arange(nx, dtype=np.float64) + 0.5) * dx
        y = (np.arange(ny, dtype=np.float64) + 0.5) * dy
        xx, yy = np.meshgrid(x, y, indexing="ij")

        def phi_f(xp, yp):
            return float(phi(float(xp), float(yp)))

        phi_grid = np.empty((nx, ny), dtype=np.float64)
        for i in range(nx):
            for j in range(ny):
                phi_grid[i, j] = phi_f(xx[i, j], yy[i, j])
        active = phi_grid <= 0.0
        if not np.any(active):
            raise ValueError("level-set contains no active material nodes")

        def normal_at(xp, yp):
            if normal is not None:
                a, b = normal(float(xp), float(yp))
                a, b = float(a), float(b)
            else:
                h = 0.5 * min(dx, dy)
                a = (phi_f(xp + h, yp) - phi_f(xp - h, yp)) / (2.0 * h)
                b = (phi_f(xp, yp + h) - phi_f(xp, yp - h)) / (2.0 * h)
            nrm = math.hypot(a, b)
            if nrm <= 1.0e-30:
                raise ValueError("zero level-set normal encountered")
            return a / nrm, b / nrm

        samples = np.linspace(0.0, 1.0, 17)
        rows = []
        for i in range(nx):
            for j in range(ny):
                if not active[i, j]:
                    continue
                x0 = float(xx[i, j])
                y0 = float(yy[i, j])
                p0 = float(phi_grid[i, j])
                for q in range(Q):
                    ii, jj = i + int(_CX[q]), j + int(_CY[q])
                    if 0 <= ii < nx and 0 <= jj < ny and bool(active[ii, jj]):
                        continue
                    x1 = x0 + float(_CX[q]) * dx
                    y1 = y0 + float(_CY[q]) * dy
                    p1 = phi_f(x1, y1)
                    if p0 <= 0.0 and p1 >= 0.0:
                        eta = _bisect(phi_f, x0, y0, x1, y1, 0.0, 1.0, root_iterations)
                    else:
                        # first sign change on 17 samples, else a half-way fallback
                        vals = [phi_f(x0 + s * (x1 - x0), y0 + s * (y1 - y0)) for s in samples]
                        idx = next((m for m in range(len(samples) - 1)
                                    if vals[m] <= 0.0 and vals[m + 1] >= 0.0), None)
                        if idx is None:
                            eta = 0.5
                        else:
                            eta = _bisect(phi_f, x0, y0, x1, y1, float(samples[idx]),
                                          float(samples[idx + 1]), root_iterations)
                    xb = x0 + eta * (x1 - x0)
                    yb = y0 + eta * (y1 - y0)
                    nxv, nyv = normal_at(xb, yb)
                    eta = float(np.clip(eta, 1.0e-6, 1.0 - 1.0e-6))
                    bid = 1 if boundary_id is None else int(boundary_id(xb, yb, nxv, nyv))
                    rows.append((i, j, q, max(0, min(MAX_BOUNDARY_IDS - 1, bid)), eta, xb, yb,
                                 nxv, nyv))
        cols = list(zip(*rows)) if rows else [()] * 9
        ints = [np.ascontiguousarray(np.asarray(c, dtype=np.int32)) for c in cols[:4]]
        reals = [np.ascontiguousarray(np.asarray(c, dtype=np.float64)) for c in cols[4:]]
        link_i, link_j, link_q, link_bid = ints
        link_eta, link_xb, link_yb, link_nx, link_ny = reals
        lsq = build_boundary_lsq_weights(
            active=active.astype(np.int32), x_coords=x, y_coords=y, link_i=link_i, link_j=link_j,
            link_xb=link_xb, link_yb=link_yb, link_nx=link_nx, link_ny=link_ny, dx=dx)
        return cls(nx=int(nx), ny=int(ny), length_x=float(length_x), length_y=float(length_y),
                   active=np.ascontiguousarray(active.astype(np.int32)), link_i=link_i,
                   link_j=link_j, link_q=link_q, link_boundary_id=link_bid, link_eta=link_eta,
                   link_xb=link_xb, link_yb=link_yb, link_nx=link_nx, link_ny=link_ny,
                   label=label, lsq_i=lsq[0], lsq_j=lsq[1], lsq_wb=lsq[2], lsq_wt=lsq[3],
                   lsq_wx=lsq[4], lsq_wy=lsq[5], lsq_valid=lsq[6])

    @classmethod
    def circle(cls, *, nx: int, ny: int, length_x: float = 1.0, length_y: float = 1.0,
               center_x: float = 0.5, center_y: float = 0.5, radius: float = 0.38):
        def normal(x, y):
            r = max(math.hypot(x - center_x, y - center_y), 1.0e-30)
            return (x - center_x) / r, (y - center_y) / r

        return cls.from_level_set(
            nx=nx, ny=ny, length_x=length_x, length_y=length_y,
            phi=lambda x, y: float(math.hypot(x - center_x, y - center_y) - radius),
            normal=normal, label=f"circle(cx={center_x},cy={center_y},r={radius})")

    @classmethod
    def annulus(cls, *, nx: int, ny: int, length_x: float = 1.0, length_y: float = 1.0,
                center_x: float = 0.5, center_y: float = 0.5, inner_radius: float = 0.18,
                outer_radius: float = 0.42):
        if not (0.0 < inner_radius < outer_radius):
            raise ValueError("annulus requires 0 < inner_radius < outer_radius")

        def radius(x, y):
            return math.hypot(x - center_x, y - center_y)

        def phi(x, y):
            r = radius(x, y)
            return max(r - outer_radius, inner_radius - r)

        def inner(r):
            return abs(r - inner_radius) <= abs(r - outer_radius)

        def normal(x, y):
            r = max(radius(x, y), 1.0e-30)
            ex, ey = (x - center_x) / r, (y - center_y) / r
            return (-ex, -ey) if inner(r) else (ex, ey)

        def boundary_id(x, y, _nx, _ny):
            return BOUNDARY_ID_INNER if inner(radius(x, y)) else BOUNDARY_ID_OUTER

        return cls.from_level_set(
            nx=nx, ny=ny, length_x=length_x, length_y=length_y, phi=phi, normal=normal,
            boundary_id=boundary_id,
            label=f"annulus(cx={center_x},cy={center_y},ri={inner_radius},ro={outer_radius})")
