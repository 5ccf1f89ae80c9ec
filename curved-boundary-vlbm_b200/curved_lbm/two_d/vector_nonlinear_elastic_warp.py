"""D2Q4x6 lattice constants, materials and host-side initialisation.

Drop-in for ``curved_lbm.two_d.vector_nonlinear_elastic_warp`` of the
reference (curved_lbm 1.0.0).  The state per node is
``U = [v_x, v_y, F_11, F_12, F_21, F_22]`` and each of the four lattice
directions E, N, W, S carries one six-component population.

The NumPy functions below build initial populations on the host, exactly as
the reference does before uploading them (reference file
``src/curved_lbm/two_d/vector_nonlinear_elastic_warp.py``, lines cited per
function).  Their array expressions keep the reference's operation order, so
the initial populations agree bit for bit.  The time step itself runs in the
CUDA library (``curved_lbm._native``); this module launches nothing.
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass
from typing import Literal

import numpy as np

Q = 4
NCOMP = 6
FQ = Q * NCOMP

MATERIAL_SVK = 0
MATERIAL_NEO_HOOKE = 1
MATERIAL_LOG_NEO_HOOKE = 2
MATERIAL_MOONEY_RIVLIN = 3
MATERIAL_YEOH = 4
MATERIAL_GENT = 5
MATERIAL_SUGIYAMA_SVK = 6

BC_PERIODIC = 0
BC_DIRICHLET = 1
BC_NEUMANN = 2

SIDE_LEFT = 0
SIDE_RIGHT = 1
SIDE_BOTTOM = 2
SIDE_TOP = 3

VALUE_ZERO = 0
VALUE_CONSTANT = 1
VALUE_RAMP = 2
VALUE_SHEAR_VELOCITY_X = 3
VALUE_WAVE_BEAM_RICKER_Y = 4
VALUE_SINE2_HOLD = 5
VALUE_AFFINE_VELOCITY = 6

SOURCE_NONE = 0
SOURCE_CONSTANT = 1
SOURCE_DAMPING = 2

PI = 3.141592653589793

_CX = np.array([1, 0, -1, 0], dtype=np.int32)
_CY = np.array([0, 1, 0, -1], dtype=np.int32)

MaterialName = Literal[
    "svk", "neo_hooke", "log_neo_hooke", "mooney_rivlin", "yeoh", "gent", "sugiyama_svk"
]
SourceName = Literal["none", "constant", "damping"]

_MATERIALS = (
    "svk",
    "neo_hooke",
    "log_neo_hooke",
    "mooney_rivlin",
    "yeoh",
    "gent",
    "sugiyama_svk",
)
_SOURCES = ("none", "constant", "damping")


def default_device() -> str:
    """Device string: ``WARP_DEVICE`` if set, else ``cuda:0`` (reference :88-94)."""
    requested = os.environ.get("WARP_DEVICE")
    return requested if requested else "cuda:0"


def material_id(name: str) -> int:
    if name in _MATERIALS:
        return _MATERIALS.index(name)
    raise ValueError(f"unsupported material model: {name}")


def material_name(mid: int) -> str:
    return _MATERIALS[mid] if 0 <= mid < len(_MATERIALS) else f"unknown_{mid}"


def source_id(name: str) -> int:
    if name in _SOURCES:
        return _SOURCES.index(name)
    raise ValueError(f"unsupported source mode: {name}")


def source_name(sid: int) -> str:
    return _SOURCES[sid] if 0 <= sid < len(_SOURCES) else f"unknown_{sid}"


@dataclass(frozen=True)
class WarpHyperelasticMaterial:
    """Compressible hyperelastic law for the 2-D Piola map (reference :175-248)."""

    model: MaterialName
    lam: float
    mu: float = 1.0
    param0: float = 0.0
    param1: float = 0.0
    param2: float = 0.0

    def __post_init__(self) -> None:
        if self.model == "mooney_rivlin" and self.param0 == 0.0 and self.param1 == 0.0:
            csum = 0.5 * self.mu
            object.__setattr__(self, "param0", 0.75 * csum)
            object.__setattr__(self, "param1", 0.25 * csum)
        elif self.model == "yeoh" and self.param0 == 0.0:
            object.__setattr__(self, "param0", 0.5 * self.mu)
        elif self.model == "gent" and self.param0 == 0.0:
            object.__setattr__(self, "param0", 50.0)

    @classmethod
    def from_poisson(
        cls,
        model: MaterialName,
        poisson: float,
        *,
        mu: float = 1.0,
        mooney_c01_fraction: float = 0.25,
        yeoh_c2: float = 0.0,
        yeoh_c3: float = 0.0,
        gent_jm: float = 50.0,
    ) -> "WarpHyperelasticMaterial":
        if abs(1.0 - 2.0 * poisson) < 1e-14:
            raise ValueError("poisson ratio too close to 1/2")
        lam = 2.0 * mu * poisson / (1.0 - 2.0 * poisson)
        if model == "mooney_rivlin":
            if not (0.0 <= mooney_c01_fraction <= 1.0):
                raise ValueError("mooney_c01_fraction must be in [0, 1]")
            csum = 0.5 * mu
            return cls(
                model=model,
                lam=lam,
                mu=mu,
                param0=(1.0 - mooney_c01_fraction) * csum,
                param1=mooney_c01_fraction * csum,
            )
        if model == "yeoh":
            return cls(model=model, lam=lam, mu=mu, param0=0.5 * mu, param1=float(yeoh_c2),
                       param2=float(yeoh_c3))
        if model == "gent":
            if gent_jm <= 0.0:
                raise ValueError("gent_jm must be positive")
            return cls(model=model, lam=lam, mu=mu, param0=float(gent_jm))
        return cls(model=model, lam=lam, mu=mu)

    @property
    def id(self) -> int:
        return material_id(self.model)

    @property
    def poisson(self) -> float:
        return self.lam / (2.0 * (self.lam + self.mu))

    def linearized_stability_ratio(self, lattice_speed: float) -> float:
        return 2.0 * math.sqrt(self.lam + 2.0 * self.mu) / float(lattice_speed)

    @property
    def params(self) -> tuple[float, float, float]:
        return float(self.param0), float(self.param1), float(self.param2)


def _first_piola_np(F: np.ndarray, material: WarpHyperelasticMaterial) -> np.ndarray:
    """First Piola stress P(F) for F of shape (2, 2, ...) (reference :486-564)."""
    F11, F12, F21, F22 = F[0, 0], F[0, 1], F[1, 0], F[1, 1]
    lam, mu = material.lam, material.mu
    P = np.empty_like(F)
    if material.model == "svk":
        C00 = F11 * F11 + F21 * F21
        C01 = F11 * F12 + F21 * F22
        C11 = F12 * F12 + F22 * F22
        E00, E01, E11 = 0.5 * (C00 - 1.0), 0.5 * C01, 0.5 * (C11 - 1.0)
        trE = E00 + E11
        S00 = lam * trE + 2.0 * mu * E00
        S01 = 2.0 * mu * E01
        S11 = lam * trE + 2.0 * mu * E11
        P[0, 0] = F11 * S00 + F12 * S01
        P[0, 1] = F11 * S01 + F12 * S11
        P[1, 0] = F21 * S00 + F22 * S01
        P[1, 1] = F21 * S01 + F22 * S11
        return P
    J = F11 * F22 - F12 * F21
    if np.any(J <= 0.0):
        raise FloatingPointError(f"non-positive deformation Jacobian: min(J)={float(np.min(J)):.6e}")
    H = np.empty_like(F)
    H[0, 0] = F22 / J
    H[0, 1] = -F21 / J
    H[1, 0] = -F12 / J
    H[1, 1] = F11 / J
    if material.model == "neo_hooke":
        return mu * (F - H) + (0.5 * lam * (J * J - 1.0)) * H
    if material.model == "log_neo_hooke":
        return mu * (F - H) + (lam * np.log(J)) * H
    F2 = F11 * F11 + F12 * F12 + F21 * F21 + F22 * F22
    I1 = F2 + 1.0
    I2 = J * J + F2
    logJ = np.log(J)
    jm23 = np.exp((-2.0 / 3.0) * logJ)
    jm43 = np.exp((-4.0 / 3.0) * logJ)
    s1 = (-2.0 / 3.0) * I1
    s2 = 2.0 * J * J - (4.0 / 3.0) * I2
    g1 = np.empty_like(F)
    g2 = np.empty_like(F)
    for (r, c), Fv in (((0, 0), F11), ((0, 1), F12), ((1, 0), F21), ((1, 1), F22)):
        g1[r, c] = jm23 * (2.0 * Fv + s1 * H[r, c])
        g2[r, c] = jm43 * (2.0 * Fv + s2 * H[r, c])
    vol = lam * logJ * H
    if material.model == "mooney_rivlin":
        return material.param0 * g1 + material.param1 * g2 + vol
    if material.model == "yeoh":
        A = jm23 * I1 - 3.0
        return (material.param0 + 2.0 * material.param1 * A + 3.0 * material.param2 * A * A) * g1 + vol
    if material.model == "gent":
        A = jm23 * I1 - 3.0
        den = 1.0 - A / material.param0
        if np.any(den <= 0.0):
            raise FloatingPointError(
                f"Gent chain limit exceeded: min(1-(I1bar-3)/Jm)={float(np.min(den)):.6e}")
        return (0.5 * material.mu / den) * g1 + vol
    if material.model == "sugiyama_svk":
        A = jm23 * I1 - 3.0
        c2 = -0.5 * material.mu
        c3 = (material.param0 + 2.0 * material.mu) / 8.0
        return (material.mu + 2.0 * c3 * A) * g1 + c2 * g2 + vol
    raise ValueError(f"unsupported material model: {material.model}")


def _flux_np(U: np.ndarray, material: WarpHyperelasticMaterial, axis: int) -> np.ndarray:
    """Flux Phi_axis(U); axis 1 is X, axis 2 is Y (reference :567-590)."""
    F = np.empty((2, 2) + U.shape[1:], dtype=np.float64)
    F[0, 0], F[0, 1], F[1, 0], F[1, 1] = U[2], U[3], U[4], U[5]
    P = _first_piola_np(F, material)
    out = np.empty_like(U)
    col = 0 if axis == 1 else 1
    out[0] = -P[0, col]
    out[1] = -P[1, col]
    out[2] = -U[0] if axis == 1 else 0.0
    out[3] = 0.0 if axis == 1 else -U[0]
    out[4] = -U[1] if axis == 1 else 0.0
    out[5] = 0.0 if axis == 1 else -U[1]
    return out


def _flux_x_np(U, material):
    return _flux_np(U, material, 1)


def _flux_y_np(U, material):
    return _flux_np(U, material, 2)


def _equilibrium_np(U: np.ndarray, material: WarpHyperelasticMaterial, lattice_speed: float):
    """feq_q = (U + (2/c)(c_qx Phi_x + c_qy Phi_y))/4 (reference :593-603)."""
    phix = _flux_np(U, material, 1)
    phiy = _flux_np(U, material, 2)
    f = np.empty((Q, NCOMP) + U.shape[1:], dtype=np.float64)
    k = 2.0 / float(lattice_speed)
    for q in range(Q):
        f[q] = 0.25 * (U + k * (_CX[q] * phix + _CY[q] * phiy))
    return f


def _source_np(U: np.ndarray, source_mode: int, source_params: np.ndarray) -> np.ndarray:
    out = np.zeros_like(U)
    params = np.asarray(source_params, dtype=np.float64)
    if source_mode == SOURCE_CONSTANT:
        out[:] = params[:NCOMP].reshape((NCOMP,) + (1,) * (U.ndim - 1))
    elif source_mode == SOURCE_DAMPING:
        out[0] = -float(params[0]) * U[0]
        out[1] = -float(params[0]) * U[1]
    elif source_mode != SOURCE_NONE:
        raise ValueError(f"unsupported source mode id: {source_mode}")
    return out


def _spatial_derivative(U: np.ndarray, spacing: float, axis: int, periodic: bool) -> np.ndarray:
    """Centred interior, second-order one-sided edge derivative (reference :620-657)."""
    h2 = 2.0 * float(spacing)
    if periodic:
        return (np.roll(U, -1, axis=axis) - np.roll(U, 1, axis=axis)) / h2
    out = np.empty_like(U)
    if U.shape[axis] < 3:
        out.fill(0.0)
        return out

    def sl(k):
        idx = [slice(None)] * U.ndim
        idx[axis] = k
        return tuple(idx)

    out[sl(slice(1, -1))] = (U[sl(slice(2, None))] - U[sl(slice(None, -2))]) / h2
    out[sl(0)] = (-3.0 * U[sl(0)] + 4.0 * U[sl(1)] - U[sl(2)]) / h2
    out[sl(-1)] = (3.0 * U[sl(-1)] - 4.0 * U[sl(-2)] + U[sl(-3)]) / h2
    return out


def _active_derivative_first_spatial(U, active, spacing, *, periodic):
    """Masked derivative along axis 1 using active neighbours only (reference :660-729)."""
    out = np.zeros_like(U)
    active = np.asarray(active, dtype=bool)
    done = np.zeros_like(active)
    h = float(spacing)
    if U.shape[1] < 2:
        return out
    if periodic:
        up1, um1 = np.roll(U, -1, axis=1), np.roll(U, 1, axis=1)
        up2, um2 = np.roll(U, -2, axis=1), np.roll(U, 2, axis=1)
        ap1, am1 = np.roll(active, -1, axis=0), np.roll(active, 1, axis=0)
        ap2, am2 = np.roll(active, -2, axis=0), np.roll(active, 2, axis=0)
        rules = (
            (active & ap1 & am1, (up1 - um1) / (2.0 * h)),
            (active & ap1 & ap2, (-3.0 * U + 4.0 * up1 - up2) / (2.0 * h)),
            (active & am1 & am2, (3.0 * U - 4.0 * um1 + um2) / (2.0 * h)),
            (active & ap1, (up1 - U) / h),
            (active & am1, (U - um1) / h),
        )
        for mask, value in rules:
            m = mask & ~done
            out[:, m] = value[:, m]
            done |= m
        return out
    if U.shape[1] >= 3:
        m = active[1:-1] & active[2:] & active[:-2]
        tmp = out[:, 1:-1]
        tmp[:, m] = ((U[:, 2:] - U[:, :-2]) / (2.0 * h))[:, m]
        done[1:-1] |= m
        m = active[:-2] & active[1:-1] & active[2:] & ~done[:-2]
        tmp = out[:, :-2]
        tmp[:, m] = ((-3.0 * U[:, :-2] + 4.0 * U[:, 1:-1] - U[:, 2:]) / (2.0 * h))[:, m]
        done[:-2] |= m
        m = active[2:] & active[1:-1] & active[:-2] & ~done[2:]
        tmp = out[:, 2:]
        tmp[:, m] = ((3.0 * U[:, 2:] - 4.0 * U[:, 1:-1] + U[:, :-2]) / (2.0 * h))[:, m]
        done[2:] |= m
    m = active[:-1] & active[1:] & ~done[:-1]
    tmp = out[:, :-1]
    tmp[:, m] = ((U[:, 1:] - U[:, :-1]) / h)[:, m]
    done[:-1] |= m
    m = active[1:] & active[:-1] & ~done[1:]
    tmp = out[:, 1:]
    tmp[:, m] = ((U[:, 1:] - U[:, :-1]) / h)[:, m]
    return out


def _masked_spatial_derivative(U, active, spacing, axis, periodic):
    if axis == 1:
        return _active_derivative_first_spatial(U, active, spacing, periodic=periodic)
    if axis == 2:
        d = _active_derivative_first_spatial(np.swapaxes(U, 1, 2), active.T, spacing,
                                             periodic=periodic)
        return np.swapaxes(d, 1, 2)
    raise ValueError("masked derivative axis must be 1 or 2")


def _flux_jvp_np(U, W, material, axis):
    """Centred finite-difference flux tangent A_axis(U) W (reference :743-756)."""
    scale = float(np.max(np.abs(W)))
    if scale == 0.0 or not np.isfinite(scale):
        return np.zeros_like(U)
    eps = 1.0e-6 / max(1.0, scale)
    for _ in range(8):
        try:
            return (_flux_np(U + eps * W, material, axis) - _flux_np(U - eps * W, material, axis)) / (2.0 * eps)
        except FloatingPointError:
            eps *= 0.25
    raise FloatingPointError(
        "failed to compute finite-difference flux tangent for second-order initialization")


def _second_order_populations_from_derivatives_np(U, Ux, Uy, material, lattice_speed, *, dt,
                                                  source_mode=SOURCE_NONE, source_params=None):
    """f = feq - dt/2 * (W + (2/c) c_q.A W)/4 with W = U_t + c c_q.grad U (reference :759-787)."""
    if source_params is None:
        source_params = np.zeros(NCOMP, dtype=np.float64)
    AxUx = _flux_jvp_np(U, Ux, material, axis=1)
    AyUy = _flux_jvp_np(U, Uy, material, axis=2)
    Ut = _source_np(U, source_mode, source_params) - (AxUx + AyUy)
    feq = _equilibrium_np(U, material, lattice_speed)
    corr = np.empty_like(feq)
    c = float(lattice_speed)
    for q in range(Q):
        cx, cy = _CX[q], _CY[q]
        Wq = Ut + c * (cx * Ux + cy * Uy)
        AxW = _flux_jvp_np(U, Wq, material, axis=1)
        AyW = _flux_jvp_np(U, Wq, material, axis=2)
        corr[q] = 0.25 * (Wq + (2.0 / c) * (cx * AxW + cy * AyW))
    return feq - 0.5 * float(dt) * corr


def _second_order_populations_np(U, material, lattice_speed, *, dx, dy, dt, periodic_x,
                                 periodic_y, source_mode=SOURCE_NONE, source_params=None):
    Ux = _spatial_derivative(U, dx, axis=1, periodic=periodic_x)
    Uy = _spatial_derivative(U, dy, axis=2, periodic=periodic_y)
    return _second_order_populations_from_derivatives_np(
        U, Ux, Uy, material, lattice_speed, dt=dt, source_mode=source_mode,
        source_params=source_params)


def _second_order_populations_masked_np(U, active, material, lattice_speed, *, dx, dy, dt,
                                        periodic_x, periodic_y, source_mode=SOURCE_NONE,
                                        source_params=None):
    """Second-order start using active-only derivatives (reference :817-847)."""
    mask = np.asarray(active, dtype=bool)
    Uw = np.array(U, dtype=np.float64, copy=True)
    Uw[:, ~mask] = 0.0
    Uw[2, ~mask] = 1.0
    Uw[5, ~mask] = 1.0
    Ux = _masked_spatial_derivative(Uw, mask, dx, axis=1, periodic=periodic_x)
    Uy = _masked_spatial_derivative(Uw, mask, dy, axis=2, periodic=periodic_y)
    return _second_order_populations_from_derivatives_np(
        Uw, Ux, Uy, material, lattice_speed, dt=dt, source_mode=source_mode,
        source_params=source_params)


def reference_grid(nx: int, ny: int, length_x: float, length_y: float):
    dx = float(length_x) / float(nx)
    dy = float(length_y) / float(ny)
    x = (np.arange(nx, dtype=np.float64) + 0.5) * dx
    y = (np.arange(ny, dtype=np.float64) + 0.5) * dy
    return np.meshgrid(x, y, indexing="ij")
