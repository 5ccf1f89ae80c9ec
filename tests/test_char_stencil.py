"""3-D characteristic stencil builders against the reference's tables.

The reference builds the fixed geometry weights of its D3Q6 local_f closure
on the host (three_d/characteristic_stencil3d.py:18-171, LAPACK solve);
the fixtures tests/golden/geo3_shell_vectorized.npz (every cut link) and
g3_shell_localf.npz (the traction links a solver selects) hold its output.
Two builders are checked against them:

* the oracle's C restatement (oracle/char_stencil3d.c), on the CPU;
* the product's CUDA kernel (cvlbm3d_build_char_stencil, one warp per link)
  through curved_lbm's build_characteristic_weights, on the GPU.

Sample indices, probe modes and probe weights must be equal; the gradient
weights come from a different linear solver than LAPACK's and must agree to
GRAD_RTOL of each link's largest weight (measured: 2.8e-14).  Both builders
raise the reference's ValueError for a link without a full-rank fit.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

import cases

GRAD_RTOL = 1e-12


def _fixture_cases(golden_dir):
    from curved_lbm import workloads
    from curved_lbm.three_d import curved_boundary_warp3d as c3

    d, cfg = cases.load(golden_dir / "geo3_shell_vectorized.npz")
    yield "geo3_shell_vectorized", workloads.shell_geometry(cfg["n"], cfg["length"], cfg["ri"],
                                                            cfg["ro"]), None, d
    d, cfg = cases.load(golden_dir / "g3_shell_localf.npz")
    g = cases.geometry_3d(cfg["geometry"])
    spec = c3.CurvedBoundarySpec3D(**cases.boundary_kwargs(cfg["boundary"]))
    ck = spec.component_kind_table(16)
    lck = ck[:, np.clip(g.link_boundary_id, 0, 15)]
    yield "g3_shell_localf", g, np.any(lck == 2, axis=0), d


def _check(name, fit, idx, w, modes):
    np.testing.assert_array_equal(fit["indices"], idx, err_msg=f"{name} indices")
    np.testing.assert_array_equal(fit["probe_modes"], modes, err_msg=f"{name} modes")
    np.testing.assert_array_equal(fit["weights"][0], w[0], err_msg=f"{name} probe weights")
    scale = np.max(np.abs(w[1:]), axis=(0, 1))
    err = np.max(np.abs(fit["weights"][1:] - w[1:]), axis=(0, 1))
    assert np.all(err <= GRAD_RTOL * scale), (name, float(np.max(err / np.maximum(scale, 1e-300))))


def _tables(g):
    from curved_lbm.three_d import geometry3d as g3

    return g3._sparse_tables_from_geometry(g)


def _deficient_geometry():
    """One cut link whose 7^3 cube holds only 8 active nodes: no quadratic fit."""
    n = 9
    active = np.zeros((n, n, n), dtype=bool)
    active[4:6, 4:6, 4:6] = True
    dx = 0.1
    link = dict(link_i=[4], link_j=[4], link_k=[4], link_q=[3], link_boundary_id=[1],
                link_eta=[0.4], link_xb=[(4 + 0.5 - 0.4) * dx], link_yb=[4.5 * dx],
                link_zb=[4.5 * dx], link_nx=[-1.0], link_ny=[0.0], link_nz=[0.0])
    g = SimpleNamespace(active=active, nx=n, ny=n, nz=n, dx=dx, dy=dx, dz=dx, n_links=1,
                        **{k: np.asarray(v, dtype=np.int32 if k in ("link_i", "link_j", "link_k",
                                                                     "link_q", "link_boundary_id")
                                         else np.float64) for k, v in link.items()})
    active_id = np.full(active.shape, -1, np.int32)
    active_id[active] = np.arange(int(active.sum()), dtype=np.int32)
    return g, {"active_id": active_id}


def test_oracle_char_stencil_matches_reference(golden_dir):
    from oracle.oracle import available, build_char_stencil

    if not available():
        pytest.skip("oracle library not built")
    for name, g, mask, d in _fixture_cases(golden_dir):
        fit = build_char_stencil(g, _tables(g), link_mask=mask)
        _check(name, fit, d["char_indices"], d["char_weights"], d["char_modes"])


def test_oracle_char_stencil_rejects_rank_deficient_fit():
    from oracle.oracle import available, build_char_stencil

    if not available():
        pytest.skip("oracle library not built")
    g, tables = _deficient_geometry()
    with pytest.raises(ValueError, match="full-rank quadratic stencil"):
        build_char_stencil(g, tables)


@pytest.mark.gpu
def test_cuda_char_stencil_matches_reference(golden_dir):
    from curved_lbm.three_d.characteristic_stencil3d import build_characteristic_weights

    for name, g, mask, d in _fixture_cases(golden_dir):
        fit = build_characteristic_weights(g, _tables(g), link_mask=mask)
        _check(name, fit, d["char_indices"], d["char_weights"], d["char_modes"])
        if mask is not None:
            assert np.array_equal(fit["link_mask"], mask)


@pytest.mark.gpu
def test_cuda_char_stencil_matches_oracle_on_shell96():
    """A 96^3 shell (tens of thousands of cut links): the CUDA and C builders
    take the same sample sets and weights (gradient weights to round-off)."""
    from curved_lbm import workloads
    from curved_lbm.three_d.characteristic_stencil3d import build_characteristic_weights
    from oracle.oracle import available, build_char_stencil

    if not available():
        pytest.skip("oracle library not built")
    g = workloads.shell_geometry(96)
    t = _tables(g)
    mask = g.link_boundary_id == 1
    ref = build_char_stencil(g, t, link_mask=mask)
    fit = build_characteristic_weights(g, t, link_mask=mask)
    _check("shell96", fit, ref["indices"], ref["weights"], ref["probe_modes"])


@pytest.mark.gpu
def test_cuda_char_stencil_rejects_rank_deficient_fit():
    from curved_lbm.three_d.characteristic_stencil3d import build_characteristic_weights

    g, tables = _deficient_geometry()
    with pytest.raises(ValueError, match="full-rank quadratic stencil"):
        build_characteristic_weights(g, tables)
