"""Batched D2Q4x6 solves (many geometries in one persistent launch per step).

GPU tests: each batched instance must equal a solo solver of the same case
after the same number of steps, bit for bit, and instances must retire on
their own residual.  CPU tests: the seeded instance table.
"""

from __future__ import annotations

import numpy as np
import pytest


def _small_batch(n_inst=3, seed=7, device="cuda:0"):
    from curved_lbm import workloads

    return workloads.superellipse_batch(n_inst, seed, device=device, n_min=36, n_max=64)


def test_instance_table_is_seeded_and_in_range():
    from curved_lbm import workloads

    a = workloads.superellipse_params(256)
    b = workloads.superellipse_params(256)
    assert a == b
    n = np.array([p["n"] for p in a])
    assert n.min() >= 96 and n.max() <= 512
    for key, lo, hi in (("p", 2, 6), ("a", 0.35, 0.5), ("b", 0.35, 0.5), ("theta", 0, np.pi),
                        ("r_in", 0.1, 0.2), ("traction", 0.01, 0.06)):
        v = np.array([p[key] for p in a])
        assert v.min() >= lo and v.max() <= hi, key


def test_instance_geometry_has_both_boundaries():
    from curved_lbm import workloads

    prm = dict(workloads.superellipse_params(1, seed=3)[0], n=48)
    g = workloads.superellipse_geometry(prm)
    ids = set(np.unique(g.link_boundary_id).tolist())
    assert ids == {1, 2}
    assert g.n_active > 0 and g.n_links > 0


@pytest.mark.gpu
def test_batched_instances_equal_solo_runs():
    import torch

    from curved_lbm.batch import BatchedCurvedBoundaryLBM2D

    _, solo = _small_batch()
    _, batched = _small_batch()
    steps = 60
    for s in solo:
        s.run(steps)
    b = BatchedCurvedBoundaryLBM2D(batched)
    b.run(steps, check_every=20, tol=0.0)  # checks on, nothing retires
    st = b.finish(refresh=False)
    torch.cuda.synchronize()
    assert (st["steps"] == steps).all()
    for a, c in zip(solo, batched):
        assert c.steps == a.steps and c.time == a.time
        assert torch.equal(a.f0, c.f0)
        assert torch.equal(a.u_star, c.u_star)


@pytest.mark.gpu
def test_batch_graph_and_autotune_keep_the_trajectory():
    import torch

    from curved_lbm.batch import BatchedCurvedBoundaryLBM2D

    _, solo = _small_batch(seed=11)
    _, batched = _small_batch(seed=11)
    b = BatchedCurvedBoundaryLBM2D(batched)
    times = b.autotune(steps=4)
    assert times and b.tile_variant in times
    g = b.graph(20)
    for _ in range(3):
        b.launch(g)
    b.finish(refresh=False)
    for s in solo:
        s.run(60)
    for a, c in zip(solo, batched):
        assert torch.equal(a.f0, c.f0)
        assert torch.equal(a.u_star, c.u_star)


@pytest.mark.gpu
def test_instances_retire_on_their_residual():
    from curved_lbm import workloads
    from curved_lbm.batch import BatchedCurvedBoundaryLBM2D

    _, batched = _small_batch(seed=5)
    b = BatchedCurvedBoundaryLBM2D(batched)
    t_min = workloads.SUPERELLIPSE_RAMP_TIME
    st = b.run_to_residual(1e-4, check_every=50, graph_steps=200, t_min=t_min,
                           max_steps=200_000)
    assert (st["status"] == 1).all(), st
    assert (st["residual"] < 1e-4).all()
    assert (st["time"] >= t_min).all()
    out = b.finish()
    for s, k in zip(batched, out["steps"]):
        assert s.steps == k
        assert not s.invalid_state()
