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
