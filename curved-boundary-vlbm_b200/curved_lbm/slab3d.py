"""Slab decomposition of one 3-D domain over several GPUs (one process each).

For lattices beyond one GPU's memory the active nodes of a
WarpSparseCurvedBoundaryLBM3D domain are split into slabs of whole x-planes
(the slowest index of the sparse raster order), balanced by active-node
count.  Slab s owns the planes [lo_s, hi_s) and also holds `halo` planes on
either side (clipped at the lattice ends).  Every slab advances its own
solver on the global lattice with only its local nodes active - cut links
and characteristic-stencil tables are taken from the global domain and
remapped to local node ids - so the arithmetic of an owned node is the
single-domain arithmetic as long as the halo covers the step's dependency
radius.  One ordered time step (collision, displacement sweep, F repair,
streaming, cut links) reads at most six layers (reference docs/method.md:
76-79: sweep 1 + gradient 2 + characteristic stencil 3), so with halo = 6
the halo is refreshed after every step: each slab receives the populations
f (72 doubles) and u* (3 doubles) of its halo nodes from their owners.
Nodes near the outer edge of a halo see a truncated lattice and compute
values that are never used before they are overwritten.

The plan (partition, local tables, exchange lists) is pure host index logic.
The exchange goes through torch.distributed point-to-point calls (NCCL
between GPUs, gloo for host arrays); slabs held by the same process copy
directly.  Owned results equal the single-domain run bit for bit.
"""

from __future__ import annotations

import dataclasses

import numpy as np

DEFAULT_HALO = 6


def slab_bounds(active: np.ndarray, n_slabs: int, halo: int = DEFAULT_HALO) -> list:
    """x-plane ranges [lo, hi) of `n_slabs` slabs with about equal active counts."""
    act = np.asarray(active, dtype=bool)
    nx = act.shape[0]
    if n_slabs < 1 or n_slabs > nx:
        raise ValueError(f"cannot split {nx} x-planes into {n_slabs} slabs")
    per = act.reshape(nx, -1).sum(axis=1).astype(np.float64)
    cum = np.concatenate([[0.0], np.cumsum(per)])
    total = cum[-1]
    cuts = [0]
    for s in range(1, n_slabs):
        c = int(np.searchsorted(cum, total * s / n_slabs, side="left"))
        c = max(c, cuts[-1] + 1)
        c = min(c, nx - (n_slabs - s))
        cuts.append(c)
    cuts.append(nx)
    return [(cuts[s], cuts[s + 1]) for s in range(n_slabs)]


class SlabPlan:
    """Partition of a 3-D geometry into x-slabs with halos (see the module docstring)."""

    def __init__(self, geometry, n_slabs: int, halo: int = DEFAULT_HALO):
        from .three_d import geometry3d as g3

        self.geometry = geometry
        self.n_slabs = int(n_slabs)
        self.halo = int(halo)
        self.tables = g3._sparse_tables_from_geometry(geometry)
        self.active_i = np.asarray(self.tables["active_i"])
        self.bounds = slab_bounds(geometry.active, self.n_slabs, self.halo)
        nx = geometry.nx
        self.local_ranges = [(max(0, lo - self.halo), min(nx, hi + self.halo))
                             for lo, hi in self.bounds]
        # global active ids of each slab's nodes, ascending (= local id order)
        self.local_nodes = [np.flatnonzero((self.active_i >= a) & (self.active_i < b))
                            for a, b in self.local_ranges]
        self.owner = np.empty(self.active_i.size, dtype=np.int32)
        for s, (lo, hi) in enumerate(self.bounds):
            self.owner[(self.active_i >= lo) & (self.active_i < hi)] = s
        link_p = np.asarray(self.tables["link_p"])
        self.local_links = [np.flatnonzero((self.active_i[link_p] >= a) & (self.active_i[link_p] < b))
                            for a, b in self.local_ranges]
        self._lists: dict = {}

    # -- per-slab geometry -------------------------------------------------
    def local_geometry(self, s: int):
        """The global geometry with only slab s's nodes active and its links."""
        g = self.geometry
        a, b = self.local_ranges[s]
        act = np.zeros_like(np.asarray(g.active, dtype=bool))
        act[a:b] = np.asarray(g.active, dtype=bool)[a:b]
        li = self.local_links[s]
        fields = {"active": act}
        for f in dataclasses.fields(g):
            if f.name.startswith("link_"):
                fields[f.name] = np.ascontiguousarray(np.asarray(getattr(g, f.name))[li])
        return dataclasses.replace(g, **fields)

    def owned(self, s: int) -> np.ndarray:
        """Boolean mask over slab s's local nodes: the nodes it owns."""
        return self.owner[self.local_nodes[s]] == s

    def local_stencil(self, s: int, stencil: dict | None):
        """Global characteristic-stencil tables restricted to slab s's links,
        node ids mapped to local ids (-1, weight 0, for a node outside the
        slab - only links of the outer halo reach that far)."""
        if stencil is None:
            return None
        glob_to_loc = np.full(self.active_i.size, -1, dtype=np.int64)
        glob_to_loc[self.local_nodes[s]] = np.arange(self.local_nodes[s].size)
        li = self.local_links[s]
        idx = np.asarray(stencil["indices"])[:, li].astype(np.int64)
        w = np.array(np.asarray(stencil["weights"])[:, :, li], dtype=np.float64)
        loc = np.where(idx >= 0, glob_to_loc[np.maximum(idx, 0)], -1)
        w[:, loc < 0] = 0.0
        return {"indices": loc.astype(np.int32), "weights": w,
                "probe_modes": np.asarray(stencil["probe_modes"])[li].astype(np.int32)}

    def exchange_lists(self, s: int) -> dict:
        """{peer: (send, recv)}: local ids (of slab s) of owned nodes that
        peer holds in its halo, and of halo nodes that peer owns, both in
        ascending global id so that the two sides pair up."""
        if s in self._lists:
            return self._lists[s]
        out = {}
        mine = self.local_nodes[s]
        pos = {int(g): k for k, g in enumerate(mine)}
        for t in range(self.n_slabs):
            if t == s:
                continue
            theirs = self.local_nodes[t]
            send_g = theirs[self.owner[theirs] == s]
            recv_g = mine[self.owner[mine] == t]
            if send_g.size or recv_g.size:
                out[t] = (np.array([pos[int(g)] for g in send_g], dtype=np.int64),
                          np.array([pos[int(g)] for g in recv_g], dtype=np.int64))
        self._lists[s] = out
        return out


# ---------------------------------------------------------------------------
# halo exchange
# ---------------------------------------------------------------------------
def _rows(state, ids):
    """(f, u*) rows of the given local nodes as one contiguous [75, k] block."""
    import torch

    f, us = state
    idx = torch.as_tensor(ids, device=f.device)
    return torch.cat([f.index_select(1, idx), us.index_select(1, idx)], dim=0).contiguous()


def _store(state, ids, block):
    import torch

    f, us = state
    idx = torch.as_tensor(ids, device=f.device)
    f.index_copy_(1, idx, block[: f.shape[0]])
    us.index_copy_(1, idx, block[f.shape[0]:])


def exchange_halos(slabs: dict, plan: SlabPlan, group=None) -> None:
    """Refresh every halo node's (f, u*) from its owner.

    `slabs` maps the slab numbers this process holds to their state pairs
    (f [72, n_local], u* [3, n_local]) as torch tensors (CUDA for NCCL, CPU
    for gloo).  Slabs held by this process copy directly; the others are
    reached by torch.distributed send/recv to rank = slab number, all pairs
    posted at once.  Every process calls this once per step.
    """
    import torch
    import torch.distributed as dist

    blocks = {}
    for s in slabs:
        for t, (send, _recv) in plan.exchange_lists(s).items():
            if send.size:
                blocks[(s, t)] = _rows(slabs[s], send)
    ops, incoming = [], []
    for s in slabs:
        for t, (_send, recv) in plan.exchange_lists(s).items():
            if not recv.size:
                continue
            if t in slabs:
                _store(slabs[s], recv, blocks[(t, s)])
            else:
                f, _ = slabs[s]
                buf = torch.empty((75, recv.size), dtype=f.dtype, device=f.device)
                ops.append(dist.P2POp(dist.irecv, buf, t, group=group))
                incoming.append((s, recv, buf))
        for t, (send, _recv) in plan.exchange_lists(s).items():
            if send.size and t not in slabs:
                ops.append(dist.P2POp(dist.isend, blocks[(s, t)], t, group=group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for s, recv, buf in incoming:
        _store(slabs[s], recv, buf)
