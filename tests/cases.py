"""Rebuild the fixture cases of ``tests/golden`` with this package.

Each fixture stores its constructor arguments as JSON (see
``tests/golden/make_golden.py``); these helpers turn them back into solver
objects of ``curved_lbm`` so the parity tests compare like with like.
"""

from __future__ import annotations

import json
import math

import numpy as np

AFFINE_A = np.array([[0.35, 0.18], [-0.10, 0.24]])
AFFINE_T = 0.20


def load(path):
    d = np.load(path)
    return d, json.loads(str(d["config"]))


def _int_keys(dct):
    return None if dct is None else {int(k): v for k, v in dct.items()}


def boundary_kwargs(spec):
    out = dict(spec)
    for key in ("id_kinds", "id_value_modes", "id_params", "id_component_kinds"):
        if key in out:
            out[key] = _int_keys(out[key])
    if out.get("id_params"):
        out["id_params"] = {k: tuple(v) for k, v in out["id_params"].items()}
    if out.get("id_component_kinds"):
        out["id_component_kinds"] = {k: tuple(v) for k, v in out["id_component_kinds"].items()}
    if out.get("component_kinds"):
        out["component_kinds"] = tuple(out["component_kinds"])
    if "params" in out:
        out["params"] = tuple(out["params"])
    return out


def geometry_2d(spec):
    from curved_lbm.two_d import curved_boundary_warp as c2

    spec = dict(spec)
    kind = spec.pop("kind")
    assert kind == "annulus"
    return c2.CurvedBoundaryGeometry.annulus(**spec)


def geometry_3d(spec):
    from curved_lbm.three_d import curved_boundary_warp3d as c3

    spec = dict(spec)
    kind = spec.pop("kind")
    if "center" in spec:
        spec["center"] = tuple(spec["center"])
    if kind == "spherical_shell":
        return c3.CurvedBoundaryGeometry3D.spherical_shell(**spec)
    return c3.CurvedBoundaryGeometry3D.sphere(**spec)


def initial_state_2d(init, geom):
    nx, ny = geom.nx, geom.ny
    U = np.zeros((6, nx, ny))
    U[2] = U[5] = 1.0
    disp = np.zeros((2, nx, ny))
    x = (np.arange(nx) + 0.5) * geom.dx
    y = (np.arange(ny) + 0.5) * geom.dy
    X, Y = np.meshgrid(x, y, indexing="ij")
    if init["kind"] == "affine":
        B = AFFINE_A / AFFINE_T
        U[0] = B[0, 0] * (X - 0.5) + B[0, 1] * (Y - 0.5)
        U[1] = B[1, 0] * (X - 0.5) + B[1, 1] * (Y - 0.5)
    elif init["kind"] == "identity_perturbed":
        U[0] = 0.01 * np.sin(3.0 * X) * np.cos(2.0 * Y)
        U[1] = -0.02 * X * Y
        U[2] = 1.0 + 0.004 * Y
        U[3] = 0.003 * X
        U[4] = -0.002 * X * Y
        U[5] = 1.0 - 0.001 * X
        disp[0] = 0.001 * X * X
        disp[1] = -0.0005 * Y
    return U, disp


def solver_2d(cfg, geom=None, **overrides):
    from curved_lbm.two_d import curved_boundary_warp as c2
    from curved_lbm.two_d.vector_nonlinear_elastic_warp import WarpHyperelasticMaterial

    geom = geom or geometry_2d(cfg["geometry"])
    m = cfg["material"]
    material = WarpHyperelasticMaterial.from_poisson(m["model"], m["poisson"], mu=m["mu"], **m.get("extra", {}))
    kw = dict(cfg["solver"])
    if "source_vector" in kw:
        kw["source_vector"] = tuple(kw["source_vector"])
    kw.update(overrides)
    return c2.WarpCurvedBoundaryLBM2D(geom, material=material,
                                      boundary=c2.CurvedBoundarySpec(**boundary_kwargs(cfg["boundary"])),
                                      **kw)


def solver_3d(cfg, geom=None, **overrides):
    from curved_lbm.three_d import curved_boundary_warp3d as c3

    geom = geom or geometry_3d(cfg["geometry"])
    m = cfg["material"]
    material = c3.WarpHyperelasticMaterial3D.from_poisson(m["model"], m["poisson"], mu=m["mu"], **m.get("extra", {}))
    kw = dict(cfg["solver"])
    kw.update(overrides)
    return c3.WarpSparseCurvedBoundaryLBM3D(
        geom, material=material, boundary=c3.CurvedBoundarySpec3D(**boundary_kwargs(cfg["boundary"])),
        **kw)
