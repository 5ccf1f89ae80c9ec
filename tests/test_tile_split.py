"""Inner / boundary tile classification of the overlapped fused 2-D step.

Runs on the CPU: the split of the annulus tile lists against a direct
restatement of its definition (no cut-link node in the tile or its 3-node
margin, no link-stencil node in the tile), and the split is a permutation of
the tile list.
"""

from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize("n", [128, 256])
def test_annulus_tile_split_matches_definition(n):
    from curved_lbm import workloads
    from curved_lbm.two_d import curved_boundary_warp as c2

    geom, _, _, _ = workloads.annulus(n)
    act = geom.active.astype(bool)
    nx, ny = act.shape
    fused = c2._fused_tables(geom, np.asarray(geom.lsq_i), np.asarray(geom.lsq_j),
                             geom.lsq_valid)
    assert fused is not None
    need = np.asarray(fused[0]).reshape(nx, ny).astype(bool)
    link = np.zeros((nx, ny), dtype=bool)
    link[geom.link_i, geom.link_j] = True
    for tile_i in (4, 8, 16):
        tiles, tj = c2._tile_list(act, tile_i)
        order, n_inner = c2._split_tiles(tiles, tj, tile_i, link, need)
        assert sorted(order.tolist()) == sorted(tiles.tolist())
        for k, t in enumerate(order.tolist()):
            i0, j0 = (t // tj) * tile_i, (t % tj) * c2.TILE_J
            region = link[max(0, i0 - 3):i0 + tile_i + 3, max(0, j0 - 3):j0 + c2.TILE_J + 3]
            own = need[i0:i0 + tile_i, j0:j0 + c2.TILE_J]
            inner = not region.any() and not own.any()
            assert inner == (k < n_inner), (tile_i, t)
        assert n_inner < len(order)
        if n >= 256:
            assert n_inner > 0
