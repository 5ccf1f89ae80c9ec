"""summary() field reductions on the device against the host NumPy reductions
of the downloaded fields (the reference's summary code): equal doubles."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host_2d(s):
    u, U, J, mask = s.displacement(), s.system_state(), s.deformation_jacobian(), s.active_mask()
    return {"max_abs_u": float(np.max(np.sqrt(np.sum(u[:, mask] * u[:, mask], axis=0)))),
            "max_abs_v": float(np.max(np.sqrt(U[0, mask] * U[0, mask] + U[1, mask] * U[1, mask]))),
            "min_J": float(np.min(J[mask])), "max_J": float(np.max(J[mask])),
            "finite": bool(np.isfinite(u[:, mask]).all() and np.isfinite(U[:, mask]).all()
                           and np.all(J[mask] > 0.0)),
            "n_active": int(np.count_nonzero(mask))}


def _host_3d(s):
    from curved_lbm.three_d.vector_nonlinear_elastic_warp3d import _det3_np

    U, u = s.U.cpu().numpy(), s.u.cpu().numpy()
    J = _det3_np(U[3:12].reshape(3, 3, s.n_active))
    return {"max_abs_u": float(np.max(np.sqrt(np.sum(u * u, axis=0)))),
            "max_abs_v": float(np.max(np.sqrt(U[0] * U[0] + U[1] * U[1] + U[2] * U[2]))),
            "min_J": float(np.min(J)), "max_J": float(np.max(J)),
            "finite": bool(np.isfinite(U).all() and np.all(J > 0))}


def test_summary_2d_matches_host_reductions():
    from curved_lbm import workloads
    from curved_lbm.two_d import curved_boundary_warp as c2

    geom, mat, spec, kw = workloads.annulus(96)
    s = c2.WarpCurvedBoundaryLBM2D(geom, material=mat, boundary=spec, device="cuda:0", **kw)
    U, disp = workloads.annulus_initial_state(96)
    s.initialize_from_numpy(U=U, displacement=disp, init_order=2)
    s.run(200)
    got = s.summary()
    for k, v in _host_2d(s).items():
        assert got[k] == v, (k, got[k], v)


def test_summary_3d_matches_host_reductions():
    from curved_lbm import workloads
    from curved_lbm.three_d import curved_boundary_warp3d as c3

    geom, mat, spec, kw = workloads.shell(32)
    s = c3.WarpSparseCurvedBoundaryLBM3D(geom, material=mat, boundary=spec, device="cuda:0", **kw)
    s.initialize_identity()
    s.run(100)
    got = s.summary()
    for k, v in _host_3d(s).items():
        assert got[k] == v, (k, got[k], v)


def test_summary_reports_non_finite_state():
    import torch

    from curved_lbm import workloads
    from curved_lbm.two_d import curved_boundary_warp as c2

    geom, mat, spec, kw = workloads.annulus(64)
    s = c2.WarpCurvedBoundaryLBM2D(geom, material=mat, boundary=spec, device="cuda:0", **kw)
    U, disp = workloads.annulus_initial_state(64)
    s.initialize_from_numpy(U=U, displacement=disp, init_order=1)
    mask = torch.as_tensor(s.active_mask(), device=s.f0.device)
    i, j = [int(v[0]) for v in np.nonzero(s.active_mask())]
    s.f0[:, i, j] = float("nan")
    got = s.summary()
    assert got["finite"] is False and np.isnan(got["min_J"]) and np.isnan(got["max_J"])
    assert bool(mask.any())
