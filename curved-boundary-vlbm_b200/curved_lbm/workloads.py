"""Synthetic benchmark workloads of the curved-boundary VLBM time step.

The first two are the reference's production traction setups at benchmark size
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

* ``affine_annulus``: D2Q4x6 affine Dirichlet annulus on [-0.55, 0.55]^2
  (stored as [0, 1.1]^2 centred at (0.55, 0.55)), r in [0.25, 0.5], both
  circles prescribing the velocity v = L X with L = [[0.01, 0.005],
  [0, -0.01]]; the reference's affine-benchmark settings (c = 10,
  omega = 2, compat_bfl, init_order 2, no source, no kinematics,
  cases/affine_annulus.py:141-166, 409-445), neo-Hooke lambda = mu = 1.
  Exact solution u = t L X, F = I + t L, v = L X (``affine_exact``).
* ``affine_convergence``: the reference's own affine convergence case
  (cases/affine_annulus.py:38-112): unit square, annulus r in [0.18, 0.42]
  centred at (0.5, 0.5), affine velocity A / T with A = [[0.35, 0.18],
  [-0.10, 0.24]], T = 0.2, neo-Hooke from Poisson ratio 0.2 and mu = 1, run
  to t = 0.2.

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


# ---------------------------------------------------------------------------
# Affine Dirichlet annulus (exact solution)
# ---------------------------------------------------------------------------
AFFINE_L = ((0.01, 0.005), (0.0, -0.01))
AFFINE_CENTER = (0.55, 0.55)


def _affine_spec(c2, B, center):
    cx, cy = center
    params = (B[0][0], B[0][1], -(B[0][0] * cx + B[0][1] * cy),
              B[1][0], B[1][1], -(B[1][0] * cx + B[1][1] * cy), 0.0, 0.0)
    params = tuple(float(v) for v in params)
    return c2.CurvedBoundarySpec(
        kind="dirichlet", value_mode=c2.CURVED_VALUE_AFFINE_VELOCITY, params=params,
        id_kinds={c2.BOUNDARY_ID_OUTER: "dirichlet", c2.BOUNDARY_ID_INNER: "dirichlet"},
        id_value_modes={c2.BOUNDARY_ID_OUTER: c2.CURVED_VALUE_AFFINE_VELOCITY,
                        c2.BOUNDARY_ID_INNER: c2.CURVED_VALUE_AFFINE_VELOCITY},
        id_params={c2.BOUNDARY_ID_OUTER: params, c2.BOUNDARY_ID_INNER: params})


_AFFINE_SOLVER = dict(lattice_speed=10.0, collision_omega=2.0, boundary_reconstruction="compat_bfl",
                      source_mode="none")


def affine_annulus(n: int = 128):
    """Affine Dirichlet annulus of the exact-solution check (module docstring)."""
    from .two_d import curved_boundary_warp as c2

    geom = c2.CurvedBoundaryGeometry.annulus(nx=n, ny=n, length_x=1.1, length_y=1.1,
                                             center_x=AFFINE_CENTER[0], center_y=AFFINE_CENTER[1],
                                             inner_radius=0.25, outer_radius=0.5)
    mat = c2.WarpHyperelasticMaterial(model="neo_hooke", lam=1.0, mu=1.0)
    return geom, mat, _affine_spec(c2, AFFINE_L, AFFINE_CENTER), dict(_AFFINE_SOLVER)


def affine_exact(geom, t: float, L=AFFINE_L, center=AFFINE_CENTER):
    """Exact (u, U) of the affine case at time t on the geometry's nodes:
    u = t L X, v = L X, F = I + t L, X measured from the annulus centre."""
    L = np.asarray(L, dtype=np.float64)
    x = (np.arange(geom.nx) + 0.5) * geom.dx - center[0]
    y = (np.arange(geom.ny) + 0.5) * geom.dy - center[1]
    X, Y = np.meshgrid(x, y, indexing="ij")
    u = np.stack([t * (L[0, 0] * X + L[0, 1] * Y), t * (L[1, 0] * X + L[1, 1] * Y)])
    U = np.zeros((6,) + X.shape)
    U[0] = L[0, 0] * X + L[0, 1] * Y
    U[1] = L[1, 0] * X + L[1, 1] * Y
    for k, (a, b) in enumerate(((0, 0), (0, 1), (1, 0), (1, 1))):
        U[2 + k] = (1.0 if a == b else 0.0) + t * L[a, b]
    return u, U


def affine_initial_state(geom, L=AFFINE_L, center=AFFINE_CENTER):
    """Start of the affine case: v = L X, F = I, u = 0 (the exact field at t = 0)."""
    _, U = affine_exact(geom, 0.0, L, center)
    return U, np.zeros((2, geom.nx, geom.ny))


AFFINE_CONV_A = ((0.35, 0.18), (-0.10, 0.24))
AFFINE_CONV_T_END = 0.20


def affine_convergence(n: int):
    """The reference's affine convergence case at grid n (module docstring)."""
    from .two_d import curved_boundary_warp as c2

    geom = c2.CurvedBoundaryGeometry.annulus(nx=n, ny=n, inner_radius=0.18, outer_radius=0.42,
                                             center_x=0.5, center_y=0.5)
    mat = c2.WarpHyperelasticMaterial.from_poisson("neo_hooke", 0.20, mu=1.0)
    B = [[a / AFFINE_CONV_T_END for a in row] for row in AFFINE_CONV_A]
    kw = dict(_AFFINE_SOLVER, local_compatibility_interval=0, local_compatibility_blend=0.05,
              local_compatibility_interior_only=True)
    return geom, mat, _affine_spec(c2, B, (0.5, 0.5)), kw


def affine_convergence_exact(geom, t: float):
    """Exact (u, U) of the convergence case: u = (t/T) A X, v = A X / T, F = I + (t/T) A."""
    A = np.asarray(AFFINE_CONV_A)
    B = A / AFFINE_CONV_T_END
    u, U = affine_exact(geom, t, B, (0.5, 0.5))
    return u, U


def affine_metrics(u, U, sigma, active, u_ex, U_ex, material, relative_l2) -> dict:
    """Relative L2 errors of the affine cases over active nodes, as the
    reference reports them (cases/affine_annulus.py:181-227)."""
    from .two_d.vector_nonlinear_elastic_warp import _first_piola_np

    F_ex = np.array([[U_ex[2].flat[0], U_ex[3].flat[0]], [U_ex[4].flat[0], U_ex[5].flat[0]]])
    P = _first_piola_np(F_ex, material)
    J = float(np.linalg.det(F_ex))
    sg = P @ F_ex.T / J
    sig_ex = np.empty_like(sigma)
    for k, (a, b) in enumerate(((0, 0), (0, 1), (1, 0), (1, 1))):
        sig_ex[k] = sg[a, b]
    F_num = U[2:6]
    F_exf = U_ex[2:6]
    I = np.zeros_like(F_exf)
    I[0] = I[3] = 1.0
    Jn = U[2] * U[5] - U[3] * U[4]
    m = np.asarray(active, dtype=bool)
    return {
        "rel_l2_u": relative_l2(u - u_ex, u_ex, m),
        "rel_l2_v": relative_l2(U[:2] - U_ex[:2], U_ex[:2], m),
        "rel_l2_F": relative_l2(F_num - F_exf, F_exf, m),
        "rel_l2_F_minus_I": relative_l2(F_num - F_exf, F_exf - I, m),
        "rel_l2_sigma": relative_l2(sigma - sig_ex, sig_ex, m),
        "min_J": float(np.min(Jn[m])),
        "max_J": float(np.max(Jn[m])),
    }


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


# ---------------------------------------------------------------------------
# Batched superellipse shells
# ---------------------------------------------------------------------------
SUPERELLIPSE_RAMP_TIME = 0.1


def superellipse_params(n_inst: int = 256, seed: int = 20261203, n_min: int = 96,
                        n_max: int = 512) -> list[dict]:
    """Seeded instance table of the batched benchmark.

    Lattice n ~ U{n_min..n_max} on [0, 1.4]^2 (the square [-0.7, 0.7]^2 centred
    at (0.7, 0.7)); outer boundary a superellipse |xi/a|^p + |eta/b|^p = 1
    rotated by theta, with p ~ U[2, 6], a, b ~ U[0.35, 0.5], theta ~ U[0, pi);
    a clamped circular hole of radius r_in ~ U[0.1, 0.2]; outer normal
    traction T ~ U[0.01, 0.06], ramped linearly over SUPERELLIPSE_RAMP_TIME.
    """
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_inst):
        out.append({"n": int(rng.integers(n_min, n_max + 1)), "p": float(rng.uniform(2.0, 6.0)),
                    "a": float(rng.uniform(0.35, 0.5)), "b": float(rng.uniform(0.35, 0.5)),
                    "theta": float(rng.uniform(0.0, math.pi)),
                    "r_in": float(rng.uniform(0.1, 0.2)),
                    "traction": float(rng.uniform(0.01, 0.06))})
    return out


def superellipse_geometry(prm: dict):
    """Level-set geometry of one batched instance (analytic normals)."""
    from .two_d import curved_boundary_warp as c2

    L, c = 1.4, 0.7
    a, b, pw, ri = prm["a"], prm["b"], prm["p"], prm["r_in"]
    ct, st = math.cos(prm["theta"]), math.sin(prm["theta"])
    split = 0.5 * (ri + min(a, b))

    def outer_phi(x, y):
        dx, dy = x - c, y - c
        xi, eta = ct * dx + st * dy, -st * dx + ct * dy
        return (abs(xi) / a) ** pw + (abs(eta) / b) ** pw - 1.0

    def phi(x, y):
        return max(outer_phi(x, y), ri - math.hypot(x - c, y - c))

    def normal(x, y):
        dx, dy = x - c, y - c
        r = math.hypot(dx, dy)
        if r < split:
            return -dx / max(r, 1e-30), -dy / max(r, 1e-30)
        xi, eta = ct * dx + st * dy, -st * dx + ct * dy
        gx = pw * math.copysign(abs(xi) ** (pw - 1.0), xi) / a ** pw
        gy = pw * math.copysign(abs(eta) ** (pw - 1.0), eta) / b ** pw
        return ct * gx - st * gy, st * gx + ct * gy

    def boundary_id(x, y, _nx, _ny):
        return 2 if math.hypot(x - c, y - c) < split else 1

    n = prm["n"]
    return c2.CurvedBoundaryGeometry.from_level_set(nx=n, ny=n, length_x=L, length_y=L, phi=phi,
                                                   normal=normal, boundary_id=boundary_id,
                                                   label="superellipse_batch")


def superellipse_case(prm: dict):
    """(material, boundary spec, solver kwargs) of one batched instance."""
    from .two_d import curved_boundary_warp as c2

    mat = c2.WarpHyperelasticMaterial(model="neo_hooke", lam=1.0, mu=1.0)
    params = (prm["traction"], SUPERELLIPSE_RAMP_TIME)
    spec = c2.CurvedBoundarySpec(kind="neumann", value_mode=105, params=params,
                                 id_kinds={1: "neumann", 2: "dirichlet"},
                                 id_value_modes={1: 105, 2: 0},
                                 id_params={1: params, 2: ()})
    _, _, _, kw = annulus(16)
    return mat, spec, kw


def superellipse_geometries(params: list[dict], processes: int | None = None) -> list:
    """Build the instance geometries, in a spawned process pool when asked."""
    if processes is None or processes <= 1 or len(params) <= 1:
        return [superellipse_geometry(p) for p in params]
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(processes) as pool:
        return pool.map(superellipse_geometry, params, chunksize=1)


def superellipse_solvers(params: list[dict], geometries: list, device=None) -> list:
    """Solvers of the given instances, initialised to the undeformed state."""
    from .two_d import curved_boundary_warp as c2

    solvers = []
    for prm, g in zip(params, geometries):
        mat, spec, kw = superellipse_case(prm)
        s = c2.WarpCurvedBoundaryLBM2D(g, material=mat, boundary=spec, device=device, **kw)
        U, disp = annulus_initial_state(prm["n"])
        s.initialize_from_numpy(U=U, displacement=disp, init_order=2)
        solvers.append(s)
    return solvers


def superellipse_batch(n_inst: int = 256, seed: int = 20261203, device=None,
                       processes: int | None = None, n_min: int = 96, n_max: int = 512):
    """(instance table, solvers) of the batched benchmark."""
    params = superellipse_params(n_inst, seed, n_min, n_max)
    geoms = superellipse_geometries(params, processes)
    return params, superellipse_solvers(params, geoms, device)


# ---------------------------------------------------------------------------
# Finite tube under end stretch and twist (warm-start data set)
# ---------------------------------------------------------------------------
TUBE_LENGTH = 2.0
TUBE_RAMP_TIME = 2.0


def tube_params(n: int, seed: int = 7, min_wall: float = 0.0) -> list[dict]:
    """Seeded tube cases: r_in ~ U[0.3, 0.5], r_out ~ U[max(0.6, r_in + min_wall), 0.9],
    stretch ~ U[1.0, 1.3] (axial end displacement (stretch - 1) * length),
    twist ~ U[0, pi/4].  `min_wall` keeps the wall several lattice cells thick
    on coarse lattices (the local_f characteristic stencil needs a full-rank
    quadratic fit within three cells); r_in is capped so that the range of
    r_out stays non-empty."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        ri = float(rng.uniform(0.3, min(0.5, 0.9 - min_wall)))
        ro = float(rng.uniform(max(0.6, ri + min_wall), 0.9))
        out.append({"r_in": ri, "r_out": ro, "stretch": float(rng.uniform(1.0, 1.3)),
                    "twist": float(rng.uniform(0.0, math.pi / 4))})
    return out


def tube_lattice(nxy: int = 32):
    """(nx, ny, nz, dx): the tube lattice, nxy^2 x 2 nxy nodes of spacing 1.92/nxy
    (x and y span 1.92 >= 2 * 0.9; z spans 3.84 around the length-2 tube)."""
    dx = 1.92 / nxy
    return nxy, nxy, 2 * nxy, dx


def tube_geometry(prm: dict, nxy: int = 32):
    """Tube r_in <= rho <= r_out, z0 <= z <= z0 + 2 on the tube lattice.

    Boundary ids as the reference's tube case (cases/tube_pull_torsion.py):
    1 outer wall, 2 inner wall (both traction free), 3 left end (clamped),
    4 right end (prescribed stretch and twist)."""
    from .three_d import curved_boundary_warp3d as c3

    nx, ny, nz, dx = tube_lattice(nxy)
    cx, cy = 0.5 * nx * dx, 0.5 * ny * dx
    z0 = 0.5 * (nz * dx - TUBE_LENGTH)
    z1 = z0 + TUBE_LENGTH
    ri, ro = prm["r_in"], prm["r_out"]

    def phiv(X, Y, Z):
        X, Y, Z = np.broadcast_arrays(X, Y, Z)
        r = np.sqrt((X - cx) ** 2 + (Y - cy) ** 2)
        return np.maximum.reduce((r - ro, ri - r, z0 - Z, Z - z1))

    def normv(X, Y, Z):
        X, Y, Z = np.broadcast_arrays(X, Y, Z)
        r = np.maximum(np.sqrt((X - cx) ** 2 + (Y - cy) ** 2), 1e-30)
        ex, ey = (X - cx) / r, (Y - cy) / r
        d = np.stack([np.abs(r - ro), np.abs(r - ri), np.abs(Z - z0), np.abs(Z - z1)])
        m = np.argmin(d, axis=0)
        nxv = np.select([m == 0, m == 1], [ex, -ex], 0.0)
        nyv = np.select([m == 0, m == 1], [ey, -ey], 0.0)
        nzv = np.select([m == 2, m == 3], [-np.ones_like(Z), np.ones_like(Z)], 0.0)
        return nxv, nyv, nzv

    def bid(x, y, z, *_):
        r = math.sqrt((x - cx) ** 2 + (y - cy) ** 2)
        d = [abs(r - ro), abs(r - ri), abs(z - z0), abs(z - z1)]
        return (1, 2, 3, 4)[int(np.argmin(d))]

    return c3.CurvedBoundaryGeometry3D.from_level_set(
        nx=nx, ny=ny, nz=nz, length_x=nx * dx, length_y=ny * dx, length_z=nz * dx,
        phi=lambda x, y, z: float(phiv(np.asarray(x), np.asarray(y), np.asarray(z))),
        boundary_id=bid, phi_vectorized=phiv, normal_vectorized=normv, label="tube")


def tube_case(prm: dict, nxy: int = 32, ramp_time: float = TUBE_RAMP_TIME):
    """(material, boundary spec, solver kwargs) of one tube case.  The right
    end follows the exact stretch + twist displacement of
    CURVED3D_VALUE_Z_STRETCH_EXACT_TWIST_VELOCITY, ramped over `ramp_time`
    (0: applied at once, as a warm start needs)."""
    from .three_d import curved_boundary_warp3d as c3

    nx, ny, _, dx = tube_lattice(nxy)
    cx, cy = 0.5 * nx * dx, 0.5 * ny * dx
    mat = c3.WarpHyperelasticMaterial3D(model="neo_hooke", lam=1.0, mu=1.0)
    right = (cx, cy, (prm["stretch"] - 1.0) * TUBE_LENGTH, prm["twist"], float(ramp_time))
    spec = c3.CurvedBoundarySpec3D(
        kind="neumann", value_mode=c3.CURVED3D_VALUE_ZERO,
        id_kinds={1: "neumann", 2: "neumann", 3: "dirichlet", 4: "dirichlet"},
        id_value_modes={1: 0, 2: 0, 3: 0, 4: c3.CURVED3D_VALUE_Z_STRETCH_EXACT_TWIST_VELOCITY},
        id_params={4: right})
    kw = dict(lattice_speed=10.0, collision_omega=1.8, boundary_reconstruction="local_f",
              source_mode="damping", damping_gamma=10.0, local_displacement_interval=1,
              local_displacement_sweeps=1, local_displacement_relax=0.85,
              local_displacement_boundary_weight=100.0, local_displacement_boundary_id=-1,
              local_compatibility_interval=1, local_compatibility_blend=0.5)
    return mat, spec, kw
