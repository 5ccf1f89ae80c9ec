"""Exact checkpoint / restart of the 2-D and 3-D solvers.

A run that writes a checkpoint and continues must end in the same state,
bit for bit, as a fresh solver that restores the checkpoint and runs the
same steps; a checkpoint from another configuration is refused.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _annulus(n):
    from curved_lbm import workloads
    from curved_lbm.two_d import curved_boundary_warp as c2

    geom, mat, spec, kw = workloads.annulus(n)
    s = c2.WarpCurvedBoundaryLBM2D(geom, material=mat, boundary=spec, **kw)
    U, disp = workloads.annulus_initial_state(n)
    s.initialize_from_numpy(U=U, displacement=disp, init_order=2)
    return s


def _shell(n):
    from curved_lbm import workloads
    from curved_lbm.three_d import curved_boundary_warp3d as c3

    geom, mat, spec, kw = workloads.shell(n)
    s = c3.WarpSparseCurvedBoundaryLBM3D(geom, material=mat, boundary=spec, **kw)
    s.initialize_identity()
    return s


def _annulus_with(n, *, traction=None, material=None, **solver_overrides):
    from curved_lbm import workloads
    from curved_lbm.two_d import curved_boundary_warp as c2

    geom, mat, spec, kw = workloads.annulus(n)
    if traction is not None:
        ramp = spec.params[1]
        spec = c2.CurvedBoundarySpec(kind="neumann", value_mode=105, params=(traction, ramp),
                                     id_kinds={1: "neumann", 2: "dirichlet"},
                                     id_value_modes={1: 105, 2: 0},
                                     id_params={1: (traction, ramp), 2: ()})
    kw.update(solver_overrides)
    return c2.WarpCurvedBoundaryLBM2D(geom, material=material or mat, boundary=spec, **kw)


def test_restore_refuses_other_load_material_or_schedule(tmp_path):
    """A checkpoint only restores into a solver whose step computes the same
    thing: another traction, material parameter, sweep relaxation or repair
    interval is refused."""
    from curved_lbm.two_d.vector_nonlinear_elastic_warp import WarpHyperelasticMaterial

    a = _annulus(96)
    a.run(4)
    a.checkpoint(tmp_path / "ck.npz")
    _annulus_with(96).restore(tmp_path / "ck.npz")  # same configuration: accepted
    others = [
        _annulus_with(96, traction=0.06),
        _annulus_with(96, material=WarpHyperelasticMaterial(model="neo_hooke", lam=1.5, mu=1.0)),
        _annulus_with(96, local_displacement_relax=0.8),
        _annulus_with(96, local_compatibility_interval=2),
        _annulus_with(96, damping_gamma=5.0),
    ]
    for s in others:
        with pytest.raises(ValueError):
            s.restore(tmp_path / "ck.npz")


def test_shell_restore_refuses_other_load(tmp_path):
    from curved_lbm import workloads
    from curved_lbm.three_d import curved_boundary_warp3d as c3

    a = _shell(24)
    a.checkpoint(tmp_path / "ck3.npz")
    geom, mat, spec, kw = workloads.shell(24)
    ramp = spec.params[1]
    other = c3.CurvedBoundarySpec3D(kind="neumann", value_mode=208, params=(0.07, ramp),
                                    id_kinds={1: "neumann", 2: "dirichlet"},
                                    id_value_modes={1: 208, 2: 0},
                                    id_params={1: (0.07, ramp), 2: ()})
    b = c3.WarpSparseCurvedBoundaryLBM3D(geom, material=mat, boundary=other, **kw)
    with pytest.raises(ValueError):
        b.restore(tmp_path / "ck3.npz")
    c = c3.WarpSparseCurvedBoundaryLBM3D(geom, material=mat, boundary=spec, **kw)
    c.restore(tmp_path / "ck3.npz")


def test_annulus_restart_is_exact(tmp_path):
    a = _annulus(160)
    a.run(30)
    a.checkpoint(tmp_path / "ck.npz")
    a.run(21)
    b = _annulus(160)
    b.restore(tmp_path / "ck.npz")
    b.run(21)
    assert (a.time, a.steps) == (b.time, b.steps)
    for k in ("f0", "u_star", "U", "u"):
        np.testing.assert_array_equal(a.numpy_field(k), b.numpy_field(k), err_msg=k)
    with pytest.raises(ValueError):
        _annulus(128).restore(tmp_path / "ck.npz")


def test_shell_restart_is_exact(tmp_path):
    a = _shell(40)
    a.run(20)
    a.checkpoint(tmp_path / "ck3.npz")
    a.run(15)
    b = _shell(40)
    b.restore(tmp_path / "ck3.npz")
    b.run(15)
    assert (a.time, a.steps) == (b.time, b.steps)
    for get in ("active_populations", "active_ustar", "active_system_state",
                "active_displacement"):
        np.testing.assert_array_equal(getattr(a, get)(), getattr(b, get)(), err_msg=get)
