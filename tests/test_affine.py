"""Affine Dirichlet annulus against its exact solution.

Two workloads (curved_lbm.workloads):

* the reference's own affine convergence case (cases/affine_annulus.py) at
  n = 64 ... 384, run to t = 0.2 with the reference's settings; its relative
  L2 errors against the exact field are published by the reference
  (validation/release_verification.json, copied to
  tests/golden/affine_published.json by make_affine_published.py).  The
  oracle (CPU) and the CUDA path (GPU, through run_until) must reproduce
  every published row to relative 1e-8 - far tighter than the reference's
  own three-significant-digit check;
* the 128^2 affine annulus on [-0.55, 0.55]^2 with v = L X on both circles,
  2000 steps: CUDA against the oracle element-wise (atol 1e-15 + rtol 1e-12)
  and both against the exact u = t L X, F = I + t L.
"""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

PUBLISHED = json.loads((GOLDEN / "affine_published.json").read_text())["rows"]
METRICS = ("rel_l2_u", "rel_l2_v", "rel_l2_F", "rel_l2_F_minus_I", "rel_l2_sigma", "min_J",
           "max_J")
METRIC_RTOL = 1e-8
RTOL, ATOL = 1e-12, 1e-15


def _check_row(got: dict, row: dict):
    for m in METRICS:
        ref = row[m]
        assert abs(got[m] - ref) <= METRIC_RTOL * abs(ref), (row["n"], m, got[m], ref)


def _close(name, got, ref):
    err = np.abs(np.asarray(got) - np.asarray(ref))
    bad = err > ATOL + RTOL * np.abs(ref)
    assert not bad.any(), f"{name}: {int(bad.sum())} entries off, max abs err {float(err.max()):.3e}"


def _oracle(geom, mat, spec, kw):
    from oracle.oracle import Oracle2D, available

    if not available():
        pytest.skip("oracle library not built")
    return Oracle2D(geom, material=mat, boundary=spec, threads=os.cpu_count() or 1, **kw)


def _oracle_run_until(o, t_end):
    # the reference's stopping rule (two_d/curved_boundary_warp.py:4296)
    while o.time < t_end - 0.5 * o.dt:
        o.step()
    o.refresh()


@pytest.mark.parametrize("row", PUBLISHED, ids=[f"n{r['n']}" for r in PUBLISHED])
def test_oracle_reproduces_published_affine_rows(row):
    from curved_lbm import workloads
    from curved_lbm.two_d.curved_boundary_warp import relative_l2

    n = row["n"]
    geom, mat, spec, kw = workloads.affine_convergence(n)
    o = _oracle(geom, mat, spec, kw)
    _, U0 = workloads.affine_convergence_exact(geom, 0.0)
    o.initialize_from_numpy(U=U0, displacement=np.zeros((2, n, n)), init_order=2)
    _oracle_run_until(o, workloads.AFFINE_CONV_T_END)
    assert o.steps == row["steps"] and o.time == row["time"]
    u_ex, U_ex = workloads.affine_convergence_exact(geom, o.time)
    got = workloads.affine_metrics(o.u, o.U, o.sigma, geom.active, u_ex, U_ex, mat, relative_l2)
    _check_row(got, row)


@pytest.mark.gpu
@pytest.mark.parametrize("row", PUBLISHED, ids=[f"n{r['n']}" for r in PUBLISHED])
def test_cuda_reproduces_published_affine_rows(row):
    """The drop-in's run_until and getters, as cases/affine_annulus.py calls them."""
    from curved_lbm import workloads
    from curved_lbm.two_d import curved_boundary_warp as c2

    n = row["n"]
    geom, mat, spec, kw = workloads.affine_convergence(n)
    s = c2.WarpCurvedBoundaryLBM2D(geom, material=mat, boundary=spec, **kw)
    _, U0 = workloads.affine_convergence_exact(geom, 0.0)
    s.initialize_from_numpy(U=U0, displacement=np.zeros((2, n, n)), init_order=2)
    s.run_until(workloads.AFFINE_CONV_T_END)
    assert s.steps == row["steps"] and s.time == row["time"]
    u_ex, U_ex = workloads.affine_convergence_exact(geom, s.time)
    got = workloads.affine_metrics(s.displacement(), s.system_state(), s.numpy_field("sigma"),
                                   s.active_mask(), u_ex, U_ex, mat, c2.relative_l2)
    _check_row(got, row)
    assert not s.invalid_state()


@pytest.mark.gpu
def test_affine_annulus_128_2000_steps():
    """128^2 affine annulus, 2000 steps: CUDA equals the oracle element-wise;
    the displacement and F - I are within 1e-5 and 1e-4 (relative L2) of the
    exact affine field (the oracle gives 4.5e-6 and 3.5e-5)."""
    from curved_lbm import workloads
    from curved_lbm.two_d import curved_boundary_warp as c2

    n, steps = 128, 2000
    geom, mat, spec, kw = workloads.affine_annulus(n)
    U0, d0 = workloads.affine_initial_state(geom)
    o = _oracle(geom, mat, spec, kw)
    o.initialize_from_numpy(U=U0, displacement=d0, init_order=2)
    o.run(steps)
    o.refresh()
    s = c2.WarpCurvedBoundaryLBM2D(geom, material=mat, boundary=spec, **kw)
    s.initialize_from_numpy(U=U0, displacement=d0, init_order=2)
    s.run(steps)
    s.refresh_current()
    assert s.steps == o.steps and s.time == o.time
    _close("f0", s.numpy_field("f0"), o.f0)
    _close("u_star", s.numpy_field("u_star"), o.u_star)
    _close("U", s.numpy_field("U"), o.U)
    _close("u", s.numpy_field("u"), o.u)
    u_ex, U_ex = workloads.affine_exact(geom, s.time)
    got = workloads.affine_metrics(s.displacement(), s.system_state(), s.numpy_field("sigma"),
                                   s.active_mask(), u_ex, U_ex, mat, c2.relative_l2)
    assert got["rel_l2_u"] < 1e-5 and got["rel_l2_F_minus_I"] < 1e-4, got
