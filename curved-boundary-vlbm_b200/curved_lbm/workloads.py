"""Synthetic benchmark workloads of the curved-boundary VLBM time step.

Both are the reference's production traction setups at benchmark size
(seeded analytic geometry, no external data):

* ``annulus``: D2Q4x6 on an n x n lattice over [0, 1.1]^2, annulus r in
  [0.25, 0.5] centred at (0.55, 0.55); inner circle clamped (boundary id 2),
  outer circle under a radial nominal traction ramped linearly 0 -> 0.05 over
  20000 steps, then held (value mode 105); c = 10, omega = 1.8, neo-Hooke
  lambda = mu = 1, local_f closure, damping gamma = 10, one displacement
  sweep (relax 0.85, boundary weight 100) and one F repair (blend 0.5) per
  step.  ``annulus(512)`` is the default benchmark.
* ``shell``: D3Q6x12 spherical shell r in [0.5, 1.0] on an n^3 lattice over
  [0, 2.2]^3, inner sphere clamped, outer sphere under a radial traction
  ramped 0 -> 0.05 over 10000 steps (value mode 208); same physics.

Each function returns ``(geometry, material, boundary_spec, solver_kwargs)``;
the solver class is the caller's choice.
"""

from __future__ import annotations

import math

import numpy as np


def annulus(n: int = 512):
    from .two_d import curved_boundary_warp as c2

    L = 1.1
    dt = (L / n) / 10.0
    ramp = 20000 * dt
    geom = c2.CurvedBoundaryGeometry.annulus(nx=n, ny=n, length_x=L, length_y=L, center_x=0.55,
                                             center_y=0.55, inner_radius=0.25, outer_radius=0.5)
    mat = c2.WarpHyperelasticMaterial(model="neo_hooke", lam=1.0, mu=1.0)
    spec = c2.CurvedBoundarySpec(kind="neumann", value_mode=105, params=(0.05, ramp),
                                 id_kinds={1: "neumann", 2: "dirichlet"},
                                 id_value_modes={1: 105, 2: 0},
                                 id_params={1: (0.05, ramp), 2: ()})
    solver = dict(lattice_speed=10.0, collision_omega=1.8, boundary_reconstruction="local_f",
                  source_mode="damping", damping_gamma=10.0, local_displacement_interval=1,
                  local_displacement_sweeps=1, local_displacement_relax=0.85,
                  local_displacement_boundary_weight=100.0, local_displacement_boundary_id=2,
                  local_compatibility_interval=1, local_compatibility_blend=0.5,
                  local_compatibility_interior_only=False)
    return geom, mat, spec, solver


def annulus_initial_state(n: int):
    """Undeformed start: F = I, zero velocity and displacement."""
    U = np.zeros((6, n, n))
    U[2] = U[5] = 1.0
    return U, np.zeros((2, n, n))


def shell_geometry(n: int = 192, L: float = 2.2, ri: float = 0.5, ro: float = 1.0):
    from .three_d import curved_boundary_warp3d as c3

    c = 0.5 * L

    def phiv(X, Y, Z):
        R = np.sqrt((X - c) ** 2 + (Y - c) ** 2 + (Z - c) ** 2)
        return np.maximum(R - ro, ri - R)

    def normv(X, Y, Z):
        X, Y, Z = np.broadcast_arrays(X, Y, Z)
        dx, dy, dz = X - c, Y - c, Z - c
        R = np.maximum(np.sqrt(dx * dx + dy * dy + dz * dz), 1e-30)
        s = np.where(np.abs(R - ri) <= np.abs(R - ro), -1.0, 1.0)
        return s * dx / R, s * dy / R, s * dz / R

    def bid(x, y, z, *_):
        r = math.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2)
        return 2 if abs(r - ri) <= abs(r - ro) else 1

    return c3.CurvedBoundaryGeometry3D.from_level_set(
        nx=n, ny=n, nz=n, length_x=L, length_y=L, length_z=L,
        phi=lambda x, y, z: float(phiv(np.asarray(x), np.asarray(y), np.asarray(z))),
        boundary_id=bid, phi_vectorized=phiv, normal_vectorized=normv, label="shell")


def shell(n: int = 192):
    from .three_d import curved_boundary_warp3d as c3

    L = 2.2
    dt = (L / n) / 10.0
    ramp = 10000 * dt
    geom = shell_geometry(n, L)
    mat = c3.WarpHyperelasticMaterial3D(model="neo_hooke", lam=1.0, mu=1.0)
    spec = c3.CurvedBoundarySpec3D(kind="neumann", value_mode=208, params=(0.05, ramp),
                                   id_kinds={1: "neumann", 2: "dirichlet"},
                                   id_value_modes={1: 208, 2: 0},
                                   id_params={1: (0.05, ramp), 2: ()})
    solver = dict(lattice_speed=10.0, collision_omega=1.8, boundary_reconstruction="local_f",
                  source_mode="damping", damping_gamma=10.0, local_displacement_interval=1,
                  local_displacement_sweeps=1, local_displacement_relax=0.85,
                  local_displacement_boundary_weight=100.0, local_displacement_boundary_id=2,
                  local_compatibility_interval=1, local_compatibility_blend=0.5)
    return geom, mat, spec, solver
