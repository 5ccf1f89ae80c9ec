"""D3Q6x12 lattice constants, materials and host-side initialisation.

Drop-in for ``curved_lbm.three_d.vector_nonlinear_elastic_warp3d`` of the
reference (curved_lbm 1.0.0).  State ``U = [v(3), F row-major (9)]``; six
directions +x, +y, +z, -x, -y, -z.  The NumPy routines restate the
reference's host functions (file ``src/curved_lbm/three_d/
vector_nonlinear_elastic_warp3d.py``, lines cited per function) in the same
operation order, so host-built initial populations agree bit for bit.  The
box solver of that file (``WarpNonlinearElasticLBM3D``) is not part of this
package.
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass
from typing import Literal, Sequence

import numpy as np

DIM = 3
Q = 6
NCOMP = 12
FQ = Q * NCOMP

MATERIAL_SVK = 0
MATERIAL_NEO_HOOKE = 1
MATERIAL_LOG_NEO_HOOKE = 2
MATERIAL_MOONEY_RIVLIN = 3
MATERIAL_YEOH = 4
MATERIAL_GENT = 5
MATERIAL_SPH_NEO_HOOKE = 6

BC_PERIODIC = 0
BC_DIRICHLET = 1
BC_NEUMANN = 2

VALUE_ZERO = 0
VALUE_CONSTANT = 1
VALUE_RAMP = 2
VALUE_SINE2_HOLD = 3
VALUE_AFFINE_VELOCITY = 4
VALUE_SHEAR_VELOCITY_X = 5

SOURCE_NONE = 0
SOURCE_CONSTANT = 1
SOURCE_DAMPING = 2

PI = 3.141592653589793

_DIRS = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1]],
                 dtype=np.int32)

MaterialName = Literal[
    "svk", "neo_hooke", "log_neo_hooke", "mooney_rivlin", "yeoh", "gent", "sph_neo_hooke"]
SourceName = Literal["none", "constant", "damping"]
_MATERIALS = ("svk", "neo_hooke", "log_neo_hooke", "mooney_rivlin", "yeoh", "gent",
              "sph_neo_hooke")
_SOURCES = ("none", "constant", "damping")


def default_device() -> str:
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
class WarpHyperelasticMaterial3D:
    """Compressible 3-D hyperelastic law (reference :188-284)."""

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
    def from_poisson(cls, model: MaterialName, poisson: float, *, mu: float = 1.0,
                     mooney_c01_fraction: float = 0.25, yeoh_c2: float = 0.0,
                     yeoh_c3: float = 0.0, gent_jm: float = 50.0):
        if abs(1.0 - 2.0 * poisson) < 1e-14:
            raise ValueError("poisson ratio too close to 1/2")
        lame = 2.0 * mu * poisson / (1.0 - 2.0 * poisson)
        lam = lame + (2.0 / 3.0) * mu if model == "sph_neo_hooke" else lame
        if model == "mooney_rivlin":
            if not (0.0 <= mooney_c01_fraction <= 1.0):
                raise ValueError("mooney_c01_fraction must be in [0, 1]")
            csum = 0.5 * mu
            return cls(model=model, lam=lam, mu=mu, param0=(1.0 - mooney_c01_fraction) * csum,
                       param1=mooney_c01_fraction * csum)
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
        lame = self.linearized_lame
        return lame / (2.0 * (lame + self.mu))

    @property
    def linearized_lame(self) -> float:
        return self.lam - (2.0 / 3.0) * self.mu if self.model == "sph_neo_hooke" else self.lam

    @property
    def bulk_modulus(self) -> float:
        return self.lam if self.model == "sph_neo_hooke" else self.lam + (2.0 / 3.0) * self.mu

    @property
    def params(self) -> tuple[float, float, float]:
        return float(self.param0), float(self.param1), float(self.param2)

    def linearized_stability_ratio(self, lattice_speed: float) -> float:
        return 2.0 * math.sqrt(self.linearized_lame + 2.0 * self.mu) / float(lattice_speed)


def _cofactor_np(F: np.ndarray) -> np.ndarray:
    """Cofactor matrix (reference :407-421)."""
    C = np.empty_like(F)
    F11, F12, F13 = F[0, 0], F[0, 1], F[0, 2]
    F21, F22, F23 = F[1, 0], F[1, 1], F[1, 2]
    F31, F32, F33 = F[2, 0], F[2, 1], F[2, 2]
    C[0, 0] = F22 * F33 - F23 * F32
    C[0, 1] = F23 * F31 - F21 * F33
    C[0, 2] = F21 * F32 - F22 * F31
    C[1, 0] = F13 * F32 - F12 * F33
    C[1, 1] = F11 * F33 - F13 * F31
    C[1, 2] = F12 * F31 - F11 * F32
    C[2, 0] = F12 * F23 - F13 * F22
    C[2, 1] = F13 * F21 - F11 * F23
    C[2, 2] = F11 * F22 - F12 * F21
    return C


def _det3_np(F: np.ndarray) -> np.ndarray:
    return (F[0, 0] * (F[1, 1] * F[2, 2] - F[1, 2] * F[2, 1])
            - F[0, 1] * (F[1, 0] * F[2, 2] - F[1, 2] * F[2, 0])
            + F[0, 2] * (F[1, 0] * F[2, 1] - F[1, 1] * F[2, 0]))


def _first_piola_np(F: np.ndarray, material: WarpHyperelasticMaterial3D) -> np.ndarray:
    """First Piola stress for F of shape (3, 3, ...) (reference :432-501)."""
    F = np.asarray(F, dtype=np.float64)
    if F.shape[:2] != (3, 3):
        raise ValueError("F must have leading shape (3,3)")
    lam, mu = material.lam, material.mu
    if material.model == "svk":
        C = np.einsum("ia...,ib...->ab...", F, F)
        E = 0.5 * C
        for k in range(3):
            E[k, k] -= 0.5
        trE = E[0, 0] + E[1, 1] + E[2, 2]
        S = 2.0 * mu * E
        for k in range(3):
            S[k, k] += lam * trE
        return np.einsum("ib...,ba...->ia...", F, S)
    J = _det3_np(F)
    if np.any(J <= 0.0):
        raise FloatingPointError(f"non-positive deformation Jacobian: min(J)={float(np.min(J)):.6e}")
    H = _cofactor_np(F) / J
    if material.model == "neo_hooke":
        return mu * (F - H) + (0.5 * lam * (J * J - 1.0)) * H
    if material.model == "log_neo_hooke":
        return mu * (F - H) + (lam * np.log(J)) * H
    C = np.einsum("ia...,ib...->ab...", F, F)
    I1 = C[0, 0] + C[1, 1] + C[2, 2]
    logJ = np.log(J)
    jm23 = np.exp((-2.0 / 3.0) * logJ)
    G1 = jm23 * (2.0 * F - (2.0 / 3.0) * I1 * H)
    if material.model == "sph_neo_hooke":
        return 0.5 * mu * G1 + (0.5 * lam * (J * J - 1.0)) * H
    trC2 = (C[0, 0] * C[0, 0] + C[1, 1] * C[1, 1] + C[2, 2] * C[2, 2]
            + 2.0 * (C[0, 1] * C[0, 1] + C[0, 2] * C[0, 2] + C[1, 2] * C[1, 2]))
    I2 = 0.5 * (I1 * I1 - trC2)
    jm43 = np.exp((-4.0 / 3.0) * logJ)
    FC = np.einsum("ib...,ba...->ia...", F, C)
    G2 = jm43 * (2.0 * (I1 * F - FC) - (4.0 / 3.0) * I2 * H)
    vol = lam * logJ * H
    if material.model == "mooney_rivlin":
        return material.param0 * G1 + material.param1 * G2 + vol
    if material.model == "yeoh":
        A = jm23 * I1 - 3.0
        return (material.param0 + 2.0 * material.param1 * A + 3.0 * material.param2 * A * A) * G1 + vol
    if material.model == "gent":
        A = jm23 * I1 - 3.0
        den = 1.0 - A / material.param0
        if np.any(den <= 0.0):
            raise FloatingPointError(f"Gent chain limit exceeded: min denom={float(np.min(den)):.6e}")
        return (0.5 * material.mu / den) * G1 + vol
    raise ValueError(f"unsupported material model: {material.model}")


def _state_to_F_np(U: np.ndarray) -> np.ndarray:
    F = np.empty((3, 3) + U.shape[1:], dtype=np.float64)
    F[0, 0], F[0, 1], F[0, 2] = U[3], U[4], U[5]
    F[1, 0], F[1, 1], F[1, 2] = U[6], U[7], U[8]
    F[2, 0], F[2, 1], F[2, 2] = U[9], U[10], U[11]
    return F


def _flux_np(U: np.ndarray, material: WarpHyperelasticMaterial3D, axis: int) -> np.ndarray:
    """Phi_axis(U) (reference :512-520)."""
    P = _first_piola_np(_state_to_F_np(U), material)
    out = np.zeros_like(U)
    for i in range(3):
        out[i] = -P[i, axis]
    for i in range(3):
        out[3 + i * 3 + axis] = -U[i]
    return out


def _speed_tuple(lattice_speed: float | Sequence[float]) -> tuple[float, float, float]:
    if np.isscalar(lattice_speed):
        v = float(lattice_speed)
        return v, v, v
    vals = tuple(float(v) for v in lattice_speed)
    if len(vals) != 3:
        raise ValueError("lattice_speed must be a scalar or a length-three sequence")
    if min(vals) <= 0.0:
        raise ValueError("all directional lattice speeds must be positive")
    return vals


def _equilibrium_np(U: np.ndarray, material: WarpHyperelasticMaterial3D,
                    lattice_speed: float | Sequence[float]) -> np.ndarray:
    """feq_q = (U + 3 sum_a s_a Phi_a / c_a)/6 (reference :535-546)."""
    fluxes = [_flux_np(U, material, a) for a in range(3)]
    speeds = _speed_tuple(lattice_speed)
    f = np.empty((Q, NCOMP) + U.shape[1:], dtype=np.float64)
    for q in range(Q):
        s = _DIRS[q]
        directional = 0
        for a in range(3):
            directional = directional + s[a] * fluxes[a] / speeds[a]
        f[q] = (1.0 / 6.0) * (U + 3.0 * directional)
    return f


def _source_np(U: np.ndarray, source_mode: int, source_params: np.ndarray) -> np.ndarray:
    out = np.zeros_like(U)
    params = np.asarray(source_params, dtype=np.float64)
    if source_mode == SOURCE_CONSTANT:
        out[:] = params[:NCOMP].reshape((NCOMP,) + (1,) * (U.ndim - 1))
    elif source_mode == SOURCE_DAMPING:
        for a in range(3):
            out[a] = -params[0] * U[a]
    elif source_mode != SOURCE_NONE:
        raise ValueError(f"unsupported source mode id: {source_mode}")
    return out


def reference_grid(nx, ny, nz, length_x, length_y, length_z):
    xs = (np.arange(nx) + 0.5) * (length_x / nx)
    ys = (np.arange(ny) + 0.5) * (length_y / ny)
    zs = (np.arange(nz) + 0.5) * (length_z / nz)
    return np.meshgrid(xs, ys, zs, indexing="ij")
