#!/usr/bin/env python3
"""Generate the golden fixtures in ``tests/golden`` from the reference itself.

Run in the build container, where the reference checkout is readable::

    python tests/golden/make_golden.py --ref-src <reference checkout>/src [--only NAME]

(or set CVLBM_REFERENCE_SRC instead of passing --ref-src)

The reference solver (``curved_lbm`` 1.0.0, Python + NVIDIA Warp 1.10.1) is
imported from its source tree with ``_warp_standin`` installed in place of
Warp, so every fixture below is produced by the reference's own geometry code,
host initialisation and kernel bodies, evaluated serially in IEEE float64.
The stand-in reproduces the reference's Warp-generated 3-D regression fixture
``tests/data/dirichlet_bfl_3d_reference.npz`` to 4e-16 (that fixture is also
copied here, unchanged, as ``dirichlet_bfl_3d_reference.npz``).

Each fixture ``<name>.npz`` stores:

* ``config``: JSON with the constructor arguments, so the tests can rebuild
  the same case with this repository's package;
* geometry tables produced by the reference (``geom_*``);
* the state right after initialisation (``f0_init``, ``ustar_init``);
* the state after ``steps`` time steps (``f0``, ``ustar``) and the refreshed
  fields the getters return (``U``, ``u``);
* for 3-D link cases, the per-link boundary data of the last step
  (``link_Fb``, ``link_Pb``, ``link_bv``, ``char_state``).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _load_reference(ref_src: str):
    sys.path.insert(0, str(HERE))
    import _warp_standin

    _warp_standin.install()
    sys.path.insert(0, ref_src)
    import curved_lbm.three_d.characteristic_stencil3d as cs3
    import curved_lbm.three_d.curved_boundary_warp3d as c3
    import curved_lbm.two_d.curved_boundary_warp as c2
    import curved_lbm.two_d.vector_nonlinear_elastic_warp as v2

    return c2, v2, c3, cs3


# ----------------------------------------------------------------------------
# Case descriptions (plain data, rebuilt by tests/conftest.py with either
# implementation).
# ----------------------------------------------------------------------------

AFFINE_A = [[0.35, 0.18], [-0.10, 0.24]]
AFFINE_T = 0.20


def affine_params(center=(0.5, 0.5)):
    cx, cy = center
    B = np.asarray(AFFINE_A) / AFFINE_T
    return [
        float(B[0, 0]),
        float(B[0, 1]),
        float(-(B[0, 0] * cx + B[0, 1] * cy)),
        float(B[1, 0]),
        float(B[1, 1]),
        float(-(B[1, 0] * cx + B[1, 1] * cy)),
        0.0,
        0.0,
    ]


CASES_2D = {
    # Dirichlet affine annulus, compat_bfl, omega=2, second-order init.
    "g2_affine_compat": dict(
        geometry=dict(kind="annulus", nx=24, ny=24, inner_radius=0.18, outer_radius=0.42),
        material=dict(model="neo_hooke", poisson=0.2, mu=1.0),
        boundary=dict(
            kind="dirichlet",
            value_mode=6,
            params=affine_params(),
            id_kinds={"1": "dirichlet", "2": "dirichlet"},
            id_value_modes={"1": 6, "2": 6},
            id_params={"1": affine_params(), "2": affine_params()},
        ),
        solver=dict(
            lattice_speed=10.0,
            collision_omega=2.0,
            boundary_reconstruction="compat_bfl",
            source_mode="none",
        ),
        init=dict(kind="affine", init_order=2),
        steps=12,
    ),
    # Traction annulus with the production local_f closure and kinematics.
    "g2_traction_localf": dict(
        geometry=dict(
            kind="annulus",
            nx=24,
            ny=24,
            length_x=1.1,
            length_y=1.1,
            center_x=0.55,
            center_y=0.55,
            inner_radius=0.25,
            outer_radius=0.5,
        ),
        material=dict(model="neo_hooke", poisson=0.2, mu=1.0),
        boundary=dict(
            kind="neumann",
            value_mode=103,
            params=[0.05, 0.02, 0.0],
            id_kinds={"1": "neumann", "2": "dirichlet"},
            id_value_modes={"1": 103, "2": 0},
            id_params={"1": [0.05, 0.02, 0.0], "2": []},
        ),
        solver=dict(
            lattice_speed=10.0,
            collision_omega=1.8,
            boundary_reconstruction="local_f",
            source_mode="damping",
            damping_gamma=10.0,
            local_compatibility_interval=1,
            local_compatibility_blend=0.5,
            local_compatibility_interior_only=False,
            local_displacement_interval=1,
            local_displacement_sweeps=1,
            local_displacement_relax=0.85,
            local_displacement_boundary_weight=100.0,
            local_displacement_boundary_id=2,
        ),
        init=dict(kind="identity", init_order=2),
        steps=12,
    ),
    # BFL predictor, constant Piola-normal traction, finite-difference Jacobian.
    "g2_bfl_mixed_fd": dict(
        geometry=dict(kind="annulus", nx=20, ny=20, inner_radius=0.2, outer_radius=0.44),
        material=dict(model="neo_hooke", poisson=0.3, mu=1.0),
        boundary=dict(
            kind="neumann",
            value_mode=101,
            params=[0.02, 0.005, 0.004, -0.01],
            id_kinds={"1": "neumann", "2": "dirichlet"},
            id_value_modes={"1": 101, "2": 1},
            id_params={"1": [0.02, 0.005, 0.004, -0.01], "2": [0.001, -0.002]},
        ),
        solver=dict(
            lattice_speed=10.0,
            collision_omega=1.7,
            boundary_reconstruction="bfl",
            source_mode="damping",
            damping_gamma=3.0,
            normal_jacobian="finite_difference",
        ),
        init=dict(kind="identity", init_order=1),
        steps=10,
    ),
    # Closed-form energy Neumann solver, masked second-order init,
    # constant source, multi-sweep and interval logic, interior-only repair.
    "g2_energy_intervals": dict(
        geometry=dict(
            kind="annulus",
            nx=22,
            ny=22,
            center_x=0.5,
            center_y=0.5,
            inner_radius=0.2,
            outer_radius=0.43,
        ),
        material=dict(model="neo_hooke", poisson=0.25, mu=1.0),
        boundary=dict(
            kind="neumann",
            value_mode=102,
            params=[0.03],
            id_kinds={"1": "neumann", "2": "dirichlet"},
            id_value_modes={"1": 102, "2": 0},
            id_params={"1": [0.03], "2": []},
        ),
        solver=dict(
            lattice_speed=10.0,
            collision_omega=1.8,
            boundary_reconstruction="local_f",
            source_mode="constant",
            source_vector=[0.001, -0.002, 0.0005, 0.0, 0.0, -0.0005],
            neumann_solver="energy",
            local_compatibility_interval=3,
            local_compatibility_blend=0.3,
            local_compatibility_interior_only=True,
            local_displacement_interval=2,
            local_displacement_sweeps=2,
            local_displacement_relax=0.7,
            local_displacement_boundary_weight=50.0,
            local_displacement_boundary_id=2,
        ),
        init=dict(kind="identity_perturbed", init_order=3),
        steps=7,
    ),
}


def _recon_case(recon: str, *, poisson=0.25, solver_extra=None, steps=10):
    """Traction (outer wall, radial pressure ramp) and clamped inner wall on a
    perturbed annulus, with the given boundary reconstruction."""
    solver = dict(lattice_speed=10.0, collision_omega=1.8, boundary_reconstruction=recon,
                  source_mode="damping", damping_gamma=5.0)
    solver.update(solver_extra or {})
    return dict(
        geometry=dict(kind="annulus", nx=24, ny=24, length_x=1.1, length_y=1.1, center_x=0.55,
                      center_y=0.55, inner_radius=0.24, outer_radius=0.49),
        material=dict(model="neo_hooke", poisson=poisson, mu=1.0),
        boundary=dict(kind="neumann", value_mode=103, params=[0.04, 0.03, 0.0],
                      id_kinds={"1": "neumann", "2": "dirichlet"},
                      id_value_modes={"1": 103, "2": 0},
                      id_params={"1": [0.04, 0.03, 0.0], "2": []}),
        solver=solver,
        init=dict(kind="identity_perturbed", init_order=2),
        steps=steps,
    )


# The remaining supported reconstructions on a traction case: the least-squares
# BFL predictor, the compatible BFL predictor with a traction wall (tangential
# image from the u stencil), the second-order characteristic closure (local_f
# plus the compatible predictor) and the single-history BFL of local_f.
CASES_2D.update({
    "g2_lsq_bfl": _recon_case("lsq_bfl"),
    "g2_compat_bfl_traction": _recon_case("compat_bfl", poisson=0.3),
    "g2_local_char2": _recon_case("local_char2"),
    "g2_local_f_bfl": _recon_case("local_f_bfl", poisson=0.2),
})

CASES_3D = {
    # Inner clamp, outer sine^2 normal traction, production local_f closure.
    "g3_shell_localf": dict(
        geometry=dict(
            kind="spherical_shell",
            nx=16,
            ny=16,
            nz=16,
            length_x=2.2,
            length_y=2.2,
            length_z=2.2,
            center=[1.1, 1.1, 1.1],
            inner_radius=0.5,
            outer_radius=1.0,
        ),
        material=dict(model="neo_hooke", poisson=0.2, mu=1.0),
        boundary=dict(
            kind="neumann",
            value_mode=203,
            params=[0.05, 0.02, 0.0],
            id_kinds={"1": "neumann", "2": "dirichlet"},
            id_value_modes={"1": 203, "2": 0},
            id_params={"1": [0.05, 0.02, 0.0], "2": []},
        ),
        solver=dict(
            lattice_speed=10.0,
            collision_omega=1.8,
            boundary_reconstruction="local_f",
            source_mode="damping",
            damping_gamma=10.0,
            local_displacement_interval=1,
            local_displacement_sweeps=1,
            local_displacement_relax=0.85,
            local_displacement_boundary_weight=100.0,
            local_compatibility_interval=1,
            local_compatibility_blend=0.5,
        ),
        init=dict(kind="identity", init_order=1),
        steps=6,
    ),
    # BFL reconstruction with Newton on the node F, finite-difference Jacobian,
    # two sweeps, repair every second step.
    "g3_shell_bfl_fd": dict(
        geometry=dict(
            kind="spherical_shell",
            nx=14,
            ny=14,
            nz=14,
            center=[0.5, 0.5, 0.5],
            inner_radius=0.2,
            outer_radius=0.44,
        ),
        material=dict(model="neo_hooke", poisson=0.25, mu=1.0),
        boundary=dict(
            kind="neumann",
            value_mode=201,
            params=[0.01, 0.002, 0.0, 0.002, -0.005, 0.001, 0.0, 0.001, 0.004],
            id_kinds={"1": "neumann", "2": "dirichlet"},
            id_value_modes={"1": 201, "2": 1},
            id_params={
                "1": [0.01, 0.002, 0.0, 0.002, -0.005, 0.001, 0.0, 0.001, 0.004],
                "2": [0.001, -0.001, 0.002],
            },
        ),
        solver=dict(
            lattice_speed=10.0,
            collision_omega=1.7,
            boundary_reconstruction="bfl",
            source_mode="damping",
            damping_gamma=2.0,
            normal_jacobian="finite_difference",
            local_displacement_interval=1,
            local_displacement_sweeps=2,
            local_displacement_boundary_weight=30.0,
            local_compatibility_interval=2,
            local_compatibility_blend=0.2,
        ),
        init=dict(kind="identity", init_order=1),
        steps=5,
    ),
    # compat_bfl: upstream extrapolation plus surface-tangent LSQ on Neumann links.
    "g3_shell_compat": dict(
        geometry=dict(
            kind="spherical_shell",
            nx=14,
            ny=14,
            nz=14,
            center=[0.5, 0.5, 0.5],
            inner_radius=0.2,
            outer_radius=0.44,
        ),
        material=dict(model="neo_hooke", poisson=0.2, mu=1.0),
        boundary=dict(
            kind="neumann",
            value_mode=202,
            params=[0.02],
            id_kinds={"1": "neumann", "2": "dirichlet"},
            id_value_modes={"1": 202, "2": 0},
            id_params={"1": [0.02], "2": []},
        ),
        solver=dict(
            lattice_speed=10.0,
            collision_omega=1.8,
            boundary_reconstruction="compat_bfl",
            source_mode="damping",
            damping_gamma=5.0,
            local_displacement_interval=1,
            local_displacement_sweeps=1,
            local_displacement_boundary_weight=100.0,
            local_compatibility_interval=1,
            local_compatibility_blend=0.5,
        ),
        init=dict(kind="identity", init_order=1),
        steps=4,
    ),
}


def _recon_case_3d(recon: str, *, poisson=0.25, steps=5):
    """Clamped inner sphere and a sin^2-ramped normal traction on the outer
    one, with the given boundary reconstruction (3-D)."""
    return dict(
        geometry=dict(kind="spherical_shell", nx=16, ny=16, nz=16, length_x=2.2, length_y=2.2,
                      length_z=2.2, center=[1.1, 1.1, 1.1], inner_radius=0.5, outer_radius=1.0),
        material=dict(model="neo_hooke", poisson=poisson, mu=1.0),
        boundary=dict(kind="neumann", value_mode=203, params=[0.04, 0.02, 0.0],
                      id_kinds={"1": "neumann", "2": "dirichlet"},
                      id_value_modes={"1": 203, "2": 0},
                      id_params={"1": [0.04, 0.02, 0.0], "2": []}),
        solver=dict(lattice_speed=10.0, collision_omega=1.8, boundary_reconstruction=recon,
                    source_mode="damping", damping_gamma=5.0, local_displacement_interval=1,
                    local_displacement_sweeps=1, local_displacement_relax=0.85,
                    local_displacement_boundary_weight=100.0, local_compatibility_interval=1,
                    local_compatibility_blend=0.5),
        init=dict(kind="identity", init_order=1),
        steps=steps,
    )


# The two 3-D reconstructions without a fixture above: half-way bounce-back
# (eta fixed at 1/2) and the single-history BFL form of local_f.
CASES_3D.update({
    "g3_shell_halfway": _recon_case_3d("halfway"),
    "g3_shell_localf_bfl": _recon_case_3d("local_f_bfl", poisson=0.3),
})

# Geometry-only pins (tables are compared bit for bit).
# One small case per material law other than neo-Hooke: the 2-D traction
# annulus (local_f closure, sweep, repair) from a perturbed state, and a 3-D
# traction shell, so that every branch of the Piola maps (and of the normal
# solves that use them) is exercised.
MATERIALS_2D = {
    "svk": {},
    "log_neo_hooke": {},
    "mooney_rivlin": {"mooney_c01_fraction": 0.3},
    "yeoh": {"yeoh_c2": 0.08, "yeoh_c3": 0.02},
    "gent": {"gent_jm": 20.0},
    "sugiyama_svk": {},
}
MATERIALS_3D = {
    "svk": {},
    "log_neo_hooke": {},
    "mooney_rivlin": {"mooney_c01_fraction": 0.3},
    "yeoh": {"yeoh_c2": 0.08, "yeoh_c3": 0.02},
    "gent": {"gent_jm": 20.0},
    "sph_neo_hooke": {},
}
for _m, _extra in MATERIALS_2D.items():
    _c = json.loads(json.dumps(CASES_2D["g2_traction_localf"]))
    _c["geometry"]["nx"] = _c["geometry"]["ny"] = 20
    _c["material"] = dict(model=_m, poisson=0.25, mu=1.0, extra=_extra)
    _c["init"] = dict(kind="identity_perturbed", init_order=2)
    _c["steps"] = 8
    CASES_2D[f"g2_mat_{_m}"] = _c
# the MRT ghost collision and the kinetic ghost filter (reference options)
for _name, _opts in (("g2_mrt_ghost", dict(collision_model="mrt_ghost", ghost_omega=1.2)),
                     ("g2_kinetic_filter", dict(kinetic_filter_strength=0.3)),
                     ("g2_mrt_filter", dict(collision_model="mrt_ghost", ghost_omega=0.9,
                                            kinetic_filter_strength=0.15))):
    _c = json.loads(json.dumps(CASES_2D["g2_traction_localf"]))
    _c["geometry"]["nx"] = _c["geometry"]["ny"] = 20
    _c["init"] = dict(kind="identity_perturbed", init_order=2)
    _c["solver"].update(_opts)
    _c["steps"] = 8
    CASES_2D[_name] = _c
# links whose displacement rows mix Dirichlet and Neumann kinds (the
# component-wise normal solve): the outer sphere with rows (N, D, N), Newton
# with the acoustic Jacobian and with finite differences, and the energy solver
for _name, _opts in (("g3_mixed_localf", {}),
                     ("g3_mixed_fd", {"normal_jacobian": "finite_difference"}),
                     ("g3_mixed_energy", {"neumann_solver": "energy"})):
    _c = json.loads(json.dumps(CASES_3D["g3_shell_localf"]))
    _c["geometry"]["nx"] = _c["geometry"]["ny"] = _c["geometry"]["nz"] = 14
    _c["boundary"].update(value_mode=1, params=[0.01, -0.02, 0.015],
                          id_value_modes={"1": 1, "2": 0},
                          id_params={"1": [0.01, -0.02, 0.015], "2": []},
                          id_component_kinds={"1": ["neumann", "dirichlet", "neumann"]})
    _c["solver"].update(_opts)
    _c["steps"] = 4
    CASES_3D[_name] = _c
for _m, _extra in MATERIALS_3D.items():
    _c = json.loads(json.dumps(CASES_3D["g3_shell_localf"]))
    _c["geometry"]["nx"] = _c["geometry"]["ny"] = _c["geometry"]["nz"] = 14
    _c["material"] = dict(model=_m, poisson=0.25, mu=1.0, extra=_extra)
    _c["steps"] = 4
    CASES_3D[f"g3_mat_{_m}"] = _c

GEOMETRY_CASES = {
    "geo2_circle_fd_normal": dict(dim=2, kind="circle_fd", nx=30, ny=30, radius=0.37),
    "geo2_superellipse": dict(
        dim=2,
        kind="superellipse",
        nx=40,
        ny=40,
        length=1.4,
        a=0.45,
        b=0.38,
        p=3.5,
        theta=0.6,
        inner_radius=0.15,
    ),
    "geo3_shell_vectorized": dict(
        dim=3, kind="shell_vectorized", n=18, length=2.2, ri=0.5, ro=1.0
    ),
}


# ----------------------------------------------------------------------------


def build_geometry_2d(c2, spec):
    spec = dict(spec)
    kind = spec.pop("kind")
    if kind == "annulus":
        return c2.CurvedBoundaryGeometry.annulus(**spec)
    raise ValueError(kind)


def build_geometry_3d(c3, spec):
    spec = dict(spec)
    kind = spec.pop("kind")
    if "center" in spec:
        spec["center"] = tuple(spec["center"])
    if kind == "spherical_shell":
        return c3.CurvedBoundaryGeometry3D.spherical_shell(**spec)
    if kind == "sphere":
        return c3.CurvedBoundaryGeometry3D.sphere(**spec)
    raise ValueError(kind)


def _int_keys(d):
    return None if d is None else {int(k): v for k, v in d.items()}


def boundary_kwargs(spec):
    out = dict(spec)
    for key in ("id_kinds", "id_value_modes", "id_params", "id_component_kinds"):
        if key in out:
            out[key] = _int_keys(out[key])
    if "id_params" in out and out["id_params"] is not None:
        out["id_params"] = {k: tuple(v) for k, v in out["id_params"].items()}
    if out.get("id_component_kinds"):
        out["id_component_kinds"] = {k: tuple(v) for k, v in out["id_component_kinds"].items()}
    if out.get("component_kinds"):
        out["component_kinds"] = tuple(out["component_kinds"])
    if "params" in out:
        out["params"] = tuple(out["params"])
    return out


def initial_state_2d(init, geometry):
    nx, ny = geometry.nx, geometry.ny
    U = np.zeros((6, nx, ny))
    U[2] = 1.0
    U[5] = 1.0
    disp = np.zeros((2, nx, ny))
    x = (np.arange(nx) + 0.5) * geometry.dx
    y = (np.arange(ny) + 0.5) * geometry.dy
    X, Y = np.meshgrid(x, y, indexing="ij")
    if init["kind"] == "affine":
        B = np.asarray(AFFINE_A) / AFFINE_T
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


def run_2d(c2, v2, name, case, out_dir):
    t0 = time.time()
    geom = build_geometry_2d(c2, case["geometry"])
    mat = case["material"]
    material = v2.WarpHyperelasticMaterial.from_poisson(mat["model"], mat["poisson"], mu=mat["mu"], **mat.get("extra", {}))
    boundary = c2.CurvedBoundarySpec(**boundary_kwargs(case["boundary"]))
    solver_kw = dict(case["solver"])
    if "source_vector" in solver_kw:
        solver_kw["source_vector"] = tuple(solver_kw["source_vector"])
    solver = c2.WarpCurvedBoundaryLBM2D(geom, material=material, boundary=boundary, **solver_kw)
    U0, disp0 = initial_state_2d(case["init"], geom)
    order = case["init"]["init_order"]
    # host-side populations exactly as initialize_from_numpy builds them
    if order == 1:
        f_host = v2._equilibrium_np(U0, material, solver.lattice_speed)
        f_host -= (0.5 * solver.dt / float(v2.Q)) * v2._source_np(
            U0, solver.source_mode, solver.source_params)[None, ...]
    elif order == 2:
        f_host = v2._second_order_populations_np(
            U0, material, solver.lattice_speed, dx=solver.dx, dy=solver.dy, dt=solver.dt,
            periodic_x=False, periodic_y=False, source_mode=solver.source_mode,
            source_params=solver.source_params)
    else:
        f_host = v2._second_order_populations_masked_np(
            U0, solver.active_np.astype(bool), material, solver.lattice_speed, dx=solver.dx,
            dy=solver.dy, dt=solver.dt, periodic_x=False, periodic_y=False,
            source_mode=solver.source_mode, source_params=solver.source_params)
    solver.initialize_from_numpy(U=U0, displacement=disp0, init_order=order)
    f0_init = solver.numpy_field("f0").copy()
    ustar_init = solver.numpy_field("u_star").copy()
    for _ in range(case["steps"]):
        solver.step()
    f0 = solver.numpy_field("f0").copy()
    ustar = solver.numpy_field("u_star").copy()
    U_step = solver.numpy_field("U").copy()
    u_step = solver.numpy_field("u").copy()
    solver.refresh_current()
    out = dict(
        config=json.dumps(dict(case, dim=2)),
        U0=U0,
        disp0=disp0,
        f_host=f_host,
        f0_init=f0_init,
        ustar_init=ustar_init,
        f0=f0,
        ustar=ustar,
        U_step=U_step,
        u_step=u_step,
        U=solver.numpy_field("U"),
        u=solver.numpy_field("u"),
        P=solver.numpy_field("P"),
        sigma=solver.numpy_field("sigma"),
        time=np.array(solver.time),
        **geometry_tables_2d(geom),
    )
    np.savez_compressed(out_dir / f"{name}.npz", **out)
    print(f"{name}: {time.time() - t0:.1f}s links={geom.n_links} active={geom.n_active}")


def geometry_tables_2d(geom):
    names = ("active", "link_i", "link_j", "link_q", "link_boundary_id", "link_eta", "link_xb",
             "link_yb", "link_nx", "link_ny", "lsq_i", "lsq_j", "lsq_wb", "lsq_wt", "lsq_wx",
             "lsq_wy", "lsq_valid")
    return {"geom_" + n: np.asarray(getattr(geom, n)) for n in names}


def geometry_tables_3d(geom):
    names = ("active", "link_i", "link_j", "link_k", "link_q", "link_boundary_id", "link_eta",
             "link_xb", "link_yb", "link_zb", "link_nx", "link_ny", "link_nz")
    return {"geom_" + n: np.asarray(getattr(geom, n)) for n in names}


def run_3d(c3, name, case, out_dir):
    t0 = time.time()
    geom = build_geometry_3d(c3, case["geometry"])
    mat = case["material"]
    material = c3.WarpHyperelasticMaterial3D.from_poisson(mat["model"], mat["poisson"], mu=mat["mu"], **mat.get("extra", {}))
    boundary = c3.CurvedBoundarySpec3D(**boundary_kwargs(case["boundary"]))
    solver = c3.WarpSparseCurvedBoundaryLBM3D(geom, material=material, boundary=boundary, **case["solver"])
    U_id = np.zeros((12, solver.n_active))
    U_id[3] = U_id[7] = U_id[11] = 1.0
    f_host = c3._equilibrium_np(U_id, material, solver.lattice_speed)
    f_host -= 0.5 * solver.dt / float(c3.Q) * solver._source_active_np(U_id)[None, ...]
    solver.initialize_identity(init_order=case["init"]["init_order"])
    f0_init = np.asarray(solver.f0.numpy()).copy()
    ustar_init = np.asarray(solver.u_star.numpy()).copy()
    for _ in range(case["steps"]):
        solver.step()
    f0 = np.asarray(solver.f0.numpy()).copy()
    ustar = np.asarray(solver.u_star.numpy()).copy()
    out = dict(
        config=json.dumps(dict(case, dim=3)),
        f_host=f_host.reshape(72, -1),
        f0_init=f0_init,
        ustar_init=ustar_init,
        f0=f0,
        ustar=ustar,
        link_Fb=np.asarray(solver.link_Fb.numpy()).copy(),
        link_Pb=np.asarray(solver.link_Pb.numpy()).copy(),
        link_bv=np.asarray(solver.link_bv.numpy()).copy(),
        char_state=np.asarray(solver.char_state.numpy()).copy(),
        time=np.array(solver.time),
        **geometry_tables_3d(geom),
    )
    if solver.characteristic_stencil is not None:
        out["char_indices"] = np.asarray(solver.characteristic_stencil["indices"])
        out["char_weights"] = np.asarray(solver.characteristic_stencil["weights"])
        out["char_modes"] = np.asarray(solver.characteristic_stencil["probe_modes"])
    if solver.tangent_lsq_active:
        out["lsq_p"] = np.asarray(solver.lsq_p.numpy())
        out["lsq_wt1"] = np.asarray(solver.lsq_wt1.numpy())
        out["lsq_wt2"] = np.asarray(solver.lsq_wt2.numpy())
        out["lsq_valid"] = np.asarray(solver.lsq_valid.numpy())
    out["neighbor"] = np.asarray(solver.neighbor.numpy())
    out["link_p"] = np.asarray(solver.link_p.numpy())
    out["link_upstream"] = np.asarray(solver.link_upstream.numpy())
    solver.refresh_current()
    out["U"] = np.asarray(solver.U.numpy()).copy()
    out["u"] = np.asarray(solver.u.numpy()).copy()
    np.savez_compressed(out_dir / f"{name}.npz", **out)
    print(f"{name}: {time.time() - t0:.1f}s links={geom.n_links} active={solver.n_active}")


def run_geometry(c2, c3, cs3, name, case, out_dir):
    t0 = time.time()
    if case["kind"] == "circle_fd":
        cx = cy = 0.5
        r = case["radius"]
        geom = c2.CurvedBoundaryGeometry.from_level_set(
            nx=case["nx"], ny=case["ny"], length_x=1.0, length_y=1.0,
            phi=lambda x, y: math.hypot(x - cx, y - cy) - r, label="circle_fd")
        out = geometry_tables_2d(geom)
    elif case["kind"] == "superellipse":
        L = case["length"]
        c = 0.5 * L
        a, b, p, th, ri = case["a"], case["b"], case["p"], case["theta"], case["inner_radius"]
        ct, st = math.cos(th), math.sin(th)

        def outer(x, y):
            xr = ct * (x - c) + st * (y - c)
            yr = -st * (x - c) + ct * (y - c)
            return (abs(xr / a) ** p + abs(yr / b) ** p) ** (1.0 / p) - 1.0

        def phi(x, y):
            return max(outer(x, y) * min(a, b), ri - math.hypot(x - c, y - c))

        def bid(x, y, _nx, _ny):
            return 2 if math.hypot(x - c, y - c) < 0.5 * (ri + min(a, b)) else 1

        geom = c2.CurvedBoundaryGeometry.from_level_set(
            nx=case["nx"], ny=case["ny"], length_x=L, length_y=L, phi=phi, boundary_id=bid,
            label="superellipse")
        out = geometry_tables_2d(geom)
    elif case["kind"] == "shell_vectorized":
        n, L, ri, ro = case["n"], case["length"], case["ri"], case["ro"]
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

        def bid(x, y, z, _a, _b, _c):
            r = math.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2)
            return 2 if abs(r - ri) <= abs(r - ro) else 1

        def phis(x, y, z):
            return float(phiv(np.asarray(x), np.asarray(y), np.asarray(z)))

        geom = c3.CurvedBoundaryGeometry3D.from_level_set(
            nx=n, ny=n, nz=n, length_x=L, length_y=L, length_z=L, phi=phis, boundary_id=bid,
            phi_vectorized=phiv, normal_vectorized=normv, label="shell_vectorized")
        out = geometry_tables_3d(geom)
        tables = c3._sparse_tables_from_geometry(geom)
        fit = cs3.build_characteristic_weights(geom, tables)
        out["char_indices"] = fit["indices"]
        out["char_weights"] = fit["weights"]
        out["char_modes"] = fit["probe_modes"]
        lsq = c3._build_sparse_tangent_lsq_weights(geom, tables)
        for k, v in lsq.items():
            out[k] = v
        out["neighbor"] = tables["neighbor"]
        out["link_p"] = tables["link_p"]
        out["link_upstream"] = tables["link_upstream"]
    else:
        raise ValueError(case["kind"])
    out["config"] = json.dumps(case)
    np.savez_compressed(out_dir / f"{name}.npz", **out)
    print(f"{name}: {time.time() - t0:.1f}s")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-src", default=os.environ.get("CVLBM_REFERENCE_SRC"),
                    help="src/ directory of the reference checkout (or CVLBM_REFERENCE_SRC)")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not args.ref_src:
        ap.error("--ref-src (or CVLBM_REFERENCE_SRC) is required")
    c2, v2, c3, cs3 = _load_reference(args.ref_src)
    out_dir = HERE
    ref_fixture = Path(args.ref_src).parent / "tests" / "data" / "dirichlet_bfl_3d_reference.npz"
    if args.only is None and ref_fixture.exists():
        shutil.copyfile(ref_fixture, out_dir / "dirichlet_bfl_3d_reference.npz")
    for name, case in GEOMETRY_CASES.items():
        if args.only in (None, name):
            run_geometry(c2, c3, cs3, name, case, out_dir)
    for name, case in CASES_2D.items():
        if args.only in (None, name):
            run_2d(c2, v2, name, case, out_dir)
    for name, case in CASES_3D.items():
        if args.only in (None, name):
            run_3d(c3, name, case, out_dir)


if __name__ == "__main__":
    main()
