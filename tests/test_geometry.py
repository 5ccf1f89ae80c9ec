"""Host geometry and initialisation against tables produced by the reference.

The fixtures were generated by the reference's own code (see
tests/golden/make_golden.py); everything compared here is exact (bit equal).
The 3-D characteristic stencil, built on the GPU, is pinned in
tests/test_char_stencil.py.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

import cases

GEO2 = ["g2_affine_compat", "g2_traction_localf", "g2_bfl_mixed_fd", "g2_energy_intervals"]
GEO3 = ["g3_shell_localf", "g3_shell_bfl_fd", "g3_shell_compat"]


def _assert_equal(name, a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (name, a.shape, b.shape)
    assert np.array_equal(a, b), (name, float(np.max(np.abs(a.astype(float) - b.astype(float)))))


@pytest.mark.parametrize("name", GEO2)
def test_annulus_tables_match_reference(golden_dir, name):
    d, cfg = cases.load(golden_dir / f"{name}.npz")
    g = cases.geometry_2d(cfg["geometry"])
    for key in d.files:
        if key.startswith("geom_"):
            _assert_equal(key, getattr(g, key[5:]), d[key])


def test_level_set_fd_normal_and_custom_ids(golden_dir):
    from curved_lbm.two_d.curved_boundary_warp import CurvedBoundaryGeometry

    d, cfg = cases.load(golden_dir / "geo2_circle_fd_normal.npz")
    r = cfg["radius"]
    g = CurvedBoundaryGeometry.from_level_set(
        nx=cfg["nx"], ny=cfg["ny"], length_x=1.0, length_y=1.0,
        phi=lambda x, y: math.hypot(x - 0.5, y - 0.5) - r)
    for key in d.files:
        if key.startswith("geom_"):
            _assert_equal(key, getattr(g, key[5:]), d[key])

    d, cfg = cases.load(golden_dir / "geo2_superellipse.npz")
    L = cfg["length"]
    c = 0.5 * L
    a, b, p, th, ri = cfg["a"], cfg["b"], cfg["p"], cfg["theta"], cfg["inner_radius"]
    ct, st = math.cos(th), math.sin(th)

    def outer(x, y):
        xr = ct * (x - c) + st * (y - c)
        yr = -st * (x - c) + ct * (y - c)
        return (abs(xr / a) ** p + abs(yr / b) ** p) ** (1.0 / p) - 1.0

    g = CurvedBoundaryGeometry.from_level_set(
        nx=cfg["nx"], ny=cfg["ny"], length_x=L, length_y=L,
        phi=lambda x, y: max(outer(x, y) * min(a, b), ri - math.hypot(x - c, y - c)),
        boundary_id=lambda x, y, _n, _m: 2 if math.hypot(x - c, y - c) < 0.5 * (ri + min(a, b)) else 1)
    for key in d.files:
        if key.startswith("geom_"):
            _assert_equal(key, getattr(g, key[5:]), d[key])


@pytest.mark.parametrize("name", GEO3)
def test_shell_tables_match_reference(golden_dir, name):
    from curved_lbm.three_d import geometry3d as g3

    d, cfg = cases.load(golden_dir / f"{name}.npz")
    g = cases.geometry_3d(cfg["geometry"])
    for key in d.files:
        if key.startswith("geom_"):
            _assert_equal(key, getattr(g, key[5:]), d[key])
    tables = g3._sparse_tables_from_geometry(g)
    for key in ("neighbor", "link_p", "link_upstream"):
        _assert_equal(key, tables[key], d[key])
    if "lsq_p" in d.files:
        lsq = g3._build_sparse_tangent_lsq_weights(g, tables)
        for key in ("lsq_p", "lsq_wt1", "lsq_wt2", "lsq_valid"):
            _assert_equal(key, lsq[key], d[key])


def test_vectorized_level_set_path(golden_dir):
    from curved_lbm.three_d import geometry3d as g3

    d, cfg = cases.load(golden_dir / "geo3_shell_vectorized.npz")
    n, L, ri, ro = cfg["n"], cfg["length"], cfg["ri"], cfg["ro"]
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

    g = g3.CurvedBoundaryGeometry3D.from_level_set(
        nx=n, ny=n, nz=n, length_x=L, length_y=L, length_z=L,
        phi=lambda x, y, z: float(phiv(np.asarray(x), np.asarray(y), np.asarray(z))),
        boundary_id=bid, phi_vectorized=phiv, normal_vectorized=normv)
    for key in d.files:
        if key.startswith("geom_"):
            _assert_equal(key, getattr(g, key[5:]), d[key])
    tables = g3._sparse_tables_from_geometry(g)
    lsq = g3._build_sparse_tangent_lsq_weights(g, tables)
    _assert_equal("lsq_wt1", lsq["lsq_wt1"], d["lsq_wt1"])


@pytest.mark.parametrize("name", GEO2)
def test_host_initial_populations_2d(golden_dir, name):
    """Equilibrium / second-order / masked second-order initial f (exact)."""
    from curved_lbm.two_d import vector_nonlinear_elastic_warp as v2

    d, cfg = cases.load(golden_dir / f"{name}.npz")
    g = cases.geometry_2d(cfg["geometry"])
    m = cfg["material"]
    mat = v2.WarpHyperelasticMaterial.from_poisson(m["model"], m["poisson"], mu=m["mu"], **m.get("extra", {}))
    s = cfg["solver"]
    c = s["lattice_speed"]
    dt = g.dx / c
    U0, _disp = cases.initial_state_2d(cfg["init"], g)
    _assert_equal("U0", U0, d["U0"])
    mode = v2.source_id(s.get("source_mode", "none"))
    sp = np.zeros(6)
    if mode == v2.SOURCE_CONSTANT:
        sp[:] = s["source_vector"]
    elif mode == v2.SOURCE_DAMPING:
        sp[0] = s["damping_gamma"]
    order = cfg["init"]["init_order"]
    if order == 1:
        f = v2._equilibrium_np(U0, mat, c)
        f -= (0.5 * dt / float(v2.Q)) * v2._source_np(U0, mode, sp)[None, ...]
    elif order == 2:
        f = v2._second_order_populations_np(U0, mat, c, dx=g.dx, dy=g.dy, dt=dt, periodic_x=False,
                                            periodic_y=False, source_mode=mode, source_params=sp)
    else:
        f = v2._second_order_populations_masked_np(U0, g.active.astype(bool), mat, c, dx=g.dx,
                                                   dy=g.dy, dt=dt, periodic_x=False,
                                                   periodic_y=False, source_mode=mode,
                                                   source_params=sp)
    _assert_equal("f_host", f, d["f_host"])


def test_host_initial_populations_3d(golden_dir):
    from curved_lbm.three_d import vector_nonlinear_elastic_warp3d as v3

    for name in GEO3:
        d, cfg = cases.load(golden_dir / f"{name}.npz")
        n = d["f_host"].shape[1]
        U = np.zeros((12, n))
        U[3] = U[7] = U[11] = 1.0
        m = cfg["material"]
        mat = v3.WarpHyperelasticMaterial3D.from_poisson(m["model"], m["poisson"], mu=m["mu"], **m.get("extra", {}))
        c = cfg["solver"]["lattice_speed"]
        g = cases.geometry_3d(cfg["geometry"])
        dt = g.dx / c
        f = v3._equilibrium_np(U, mat, c)
        src = np.zeros_like(U)
        if cfg["solver"].get("source_mode") == "damping":
            for a in range(3):
                src[a] = -cfg["solver"]["damping_gamma"] * U[a]
        f -= 0.5 * dt / float(v3.Q) * src[None, ...]
        _assert_equal(name, f.reshape(72, n), d["f_host"])
