"""Slab decomposition of one 3-D domain (curved_lbm.slab3d).

A 24^3 spherical shell of the 3-D benchmark physics (local_f traction
closure, displacement sweep, F repair) is split into x-slabs with 6-plane
halos; each slab steps on its own nodes and refreshes its halo (f, u*) from
the owners after every step.  The owned nodes must equal the single-domain
run bit for bit:

* CPU, oracle arithmetic: two gloo ranks (one slab each, exchange through
  torch.distributed send/recv), and three slabs in one process (direct
  copies);
* GPU, the CUDA solver: two slabs in one process on one device.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

N_SHELL, STEPS = 24, 12


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shell_case():
    from curved_lbm import workloads

    return workloads.shell(N_SHELL)


def _neumann_mask(geom, spec):
    from curved_lbm.three_d import curved_boundary_warp3d as c3

    ck = spec.component_kind_table(c3.MAX_BOUNDARY_IDS)
    lck = ck[:, np.clip(geom.link_boundary_id, 0, c3.MAX_BOUNDARY_IDS - 1)]
    return np.any(lck == c3.BC_NEUMANN, axis=0)


def _oracle_global(steps):
    from oracle.oracle import Oracle3D

    geom, mat, spec, kw = _shell_case()
    o = Oracle3D(geom, material=mat, boundary=spec, threads=2, **kw)
    o.initialize_identity()
    o.run(steps)
    return o


def _oracle_slabs(plan, slabs, geom, mat, spec, kw):
    from oracle.oracle import Oracle3D, build_char_stencil

    glob = build_char_stencil(geom, plan.tables, link_mask=_neumann_mask(geom, spec))
    out = {}
    for s in slabs:
        o = Oracle3D(plan.local_geometry(s), material=mat, boundary=spec, threads=2,
                     char_stencil=plan.local_stencil(s, glob), **kw)
        out[s] = o
    return out


def _state(o):
    import torch

    return (torch.from_numpy(o.f0), torch.from_numpy(o.u_star))


def _run_oracle_slabs(plan, slabs, steps, group_exchange):
    geom, mat, spec, kw = _shell_case()
    ors = _oracle_slabs(plan, slabs, geom, mat, spec, kw)
    for o in ors.values():
        o.initialize_identity()
    group_exchange({s: _state(o) for s, o in ors.items()})
    for _ in range(steps):
        for o in ors.values():
            o.step()
        group_exchange({s: _state(o) for s, o in ors.items()})
    return ors


def _gather(plan, ors):
    """Owned (global id, f, u*) of the given slabs."""
    out = []
    for s, o in ors.items():
        own = plan.owned(s)
        out.append((plan.local_nodes[s][own], o.f0[:, own].copy(), o.u_star[:, own].copy()))
    return out


def test_plan_partitions_the_domain_and_pairs_the_exchange():
    from curved_lbm import slab3d

    geom, _, _, _ = _shell_case()
    plan = slab3d.SlabPlan(geom, 3)
    n = plan.active_i.size
    owned = np.concatenate([plan.local_nodes[s][plan.owned(s)] for s in range(3)])
    assert np.array_equal(np.sort(owned), np.arange(n))
    for s in range(3):
        for t, (send, recv) in plan.exchange_lists(s).items():
            send_t, recv_t = plan.exchange_lists(t)[s]
            assert np.array_equal(plan.local_nodes[s][send], plan.local_nodes[t][recv_t])
            assert np.array_equal(plan.local_nodes[s][recv], plan.local_nodes[t][send_t])
            assert np.all(plan.owner[plan.local_nodes[s][recv]] == t)
    lo, hi = zip(*plan.bounds)
    assert lo[0] == 0 and hi[-1] == geom.nx and all(h == l for h, l in zip(hi[:-1], lo[1:]))


def test_three_slabs_in_one_process_equal_single_domain():
    from curved_lbm import slab3d

    ref = _oracle_global(STEPS)
    geom, _, _, _ = _shell_case()
    plan = slab3d.SlabPlan(geom, 3)
    ors = _run_oracle_slabs(plan, [0, 1, 2], STEPS, lambda st: slab3d.exchange_halos(st, plan))
    for gid, f, us in _gather(plan, ors):
        np.testing.assert_array_equal(f, ref.f0[:, gid])
        np.testing.assert_array_equal(us, ref.u_star[:, gid])


def _slab_worker(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from curved_lbm import replicas, slab3d

    replicas.init(backend="gloo", timeout_s=120.0)
    try:
        geom, _, _, _ = _shell_case()
        plan = slab3d.SlabPlan(geom, world)
        ors = _run_oracle_slabs(plan, [rank], STEPS, lambda st: slab3d.exchange_halos(st, plan))
        out[rank] = _gather(plan, ors)
    finally:
        replicas.finalize()


def test_two_gloo_ranks_equal_single_domain():
    import torch.multiprocessing as mp

    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_slab_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    ref = _oracle_global(STEPS)
    seen = 0
    for r in (0, 1):
        for gid, f, us in res[r]:
            np.testing.assert_array_equal(f, ref.f0[:, gid])
            np.testing.assert_array_equal(us, ref.u_star[:, gid])
            seen += gid.size
    assert seen == ref.N


@pytest.mark.gpu
def test_cuda_slabs_equal_single_domain():
    """Two slabs in one process on one device, CUDA solver, halo refreshed by
    direct copies after every step: the owned nodes equal the one-domain run."""
    from curved_lbm import slab3d
    from curved_lbm.three_d import curved_boundary_warp3d as c3
    from curved_lbm.three_d.characteristic_stencil3d import build_characteristic_weights

    geom, mat, spec, kw = _shell_case()
    whole = c3.WarpSparseCurvedBoundaryLBM3D(geom, material=mat, boundary=spec, **kw)
    whole.initialize_identity()
    whole.run(STEPS)
    plan = slab3d.SlabPlan(geom, 2)
    glob = build_characteristic_weights(geom, plan.tables, link_mask=_neumann_mask(geom, spec))
    slabs = {s: c3.WarpSparseCurvedBoundaryLBM3D(plan.local_geometry(s), material=mat,
                                                   boundary=spec,
                                                   characteristic_stencil=plan.local_stencil(s, glob),
                                                   **kw) for s in range(2)}
    for sv in slabs.values():
        sv.initialize_identity()
    slab3d.exchange_halos({s: (sv.f0, sv.u_star) for s, sv in slabs.items()}, plan)
    for _ in range(STEPS):
        for sv in slabs.values():
            sv.run(1)
        slab3d.exchange_halos({s: (sv.f0, sv.u_star) for s, sv in slabs.items()}, plan)
    f_ref, us_ref = whole.active_populations(), whole.active_ustar()
    for s, sv in slabs.items():
        own = plan.owned(s)
        gid = plan.local_nodes[s][own]
        np.testing.assert_array_equal(sv.active_populations()[:, own], f_ref[:, gid])
        np.testing.assert_array_equal(sv.active_ustar()[:, own], us_ref[:, gid])
