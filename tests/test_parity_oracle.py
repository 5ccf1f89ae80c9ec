"""CUDA time step against the CPU oracle on the benchmark workloads.

The golden fixtures are small (tens of nodes across); these cases run the
benchmark physics (traction annulus, spherical shell) on grids with many
tiles in both directions and sizes that are not multiples of the tile, and
compare with the oracle - the C restatement of the reference kernels, itself
pinned to every fixture:

* the 2-D benchmark itself (annulus512, 127,612 active nodes) for 1000
  steps, and 100^2 / 200^2 (every tile variant) for 1000 steps;
* a 64^3 spherical shell (90,240 active nodes) for 1000 steps, and 40^3 for
  200 steps with every collide variant.

Tolerance, element by element on populations, u*, U (velocity and F) and u:
|got - ref| <= 1e-15 + 1e-12 |ref|.  The kernels keep the reference's
operation order (and are built without FMA contraction), so the states
agree to round-off; the absolute floor only matters for entries that are
exactly zero in one of them.

Size-independent properties at 512^2: every fused tile shape and the
per-phase kernels give bitwise-identical states, the link overlap and a
CUDA-graph replay equal the plain run.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12
ATOL = 1e-15
THREADS = os.cpu_count() or 1


def close_rel(name, got, ref, rtol=RTOL, atol=ATOL):
    """Element-wise |got - ref| <= atol + rtol |ref|."""
    got, ref = np.asarray(got), np.asarray(ref)
    assert got.shape == ref.shape, (name, got.shape, ref.shape)
    assert np.isfinite(ref).all(), name
    err = np.abs(got - ref)
    bad = err > atol + rtol * np.abs(ref)
    assert not bad.any(), (f"{name}: {int(bad.sum())} entries off, max abs err "
                           f"{float(err.max()):.3e}, max |ref| {float(np.abs(ref).max()):.3e}")


_cache: dict = {}


def _oracle_annulus(n, steps):
    key = ("annulus", n, steps)
    if key not in _cache:
        from curved_lbm import workloads
        from oracle.oracle import Oracle2D, available

        if not available():
            pytest.skip("oracle library not built")
        geom, mat, spec, kw = workloads.annulus(n)
        o = Oracle2D(geom, material=mat, boundary=spec, threads=THREADS, **kw)
        U, disp = workloads.annulus_initial_state(n)
        o.initialize_from_numpy(U=U, displacement=disp, init_order=2)
        o.run(steps)
        _cache[key] = {k: np.array(getattr(o, k)) for k in ("f0", "u_star", "U", "u")}
    return _cache[key]


def _gpu_annulus(n, variant=None, fused=True, graphs=False):
    from curved_lbm import workloads
    from curved_lbm.two_d import curved_boundary_warp as c2

    geom, mat, spec, kw = workloads.annulus(n)
    s = c2.WarpCurvedBoundaryLBM2D(geom, material=mat, boundary=spec, **kw)
    s.use_graphs = graphs  # run() on the plain launch path unless asked
    if variant is not None:
        s._select_variant(variant)
    s._set_fused(fused)
    U, disp = workloads.annulus_initial_state(n)
    s.initialize_from_numpy(U=U, displacement=disp, init_order=2)
    return s


@pytest.mark.parametrize("n", [100, 200])
def test_annulus_1000_steps_match_oracle(n):
    ref = _oracle_annulus(n, 1000)
    s = _gpu_annulus(n)
    s.run(1000)
    for k in ("f0", "u_star", "U", "u"):
        close_rel(k, s.numpy_field(k), ref[k])


def test_annulus512_1000_steps_match_oracle():
    """The benchmark configuration itself (512^2, 127,612 active nodes, 2,792
    cut links) with the solver's default path: autotuned tile shape, link
    overlap on, run() through cached CUDA graphs."""
    ref = _oracle_annulus(512, 1000)
    s = _gpu_annulus(512, graphs=True)
    s.autotune(steps=10)
    s.run(1000)
    for k in ("f0", "u_star", "U", "u"):
        close_rel(k, s.numpy_field(k), ref[k])
    _cache.pop(("annulus", 512, 1000), None)


@pytest.mark.parametrize("variant", list(range(11)))
def test_annulus_tile_variants_match_oracle(variant):
    ref = _oracle_annulus(200, 1000)
    s = _gpu_annulus(200, variant=variant)
    s.run(1000)
    for k in ("f0", "u_star", "U", "u"):
        close_rel(k, s.numpy_field(k), ref[k])


def _oracle_shell(n, steps, stencil=None):
    """Oracle replay of the shell; `stencil`: the characteristic stencil
    tables the CUDA solver built, so both step on identical inputs (the
    builders themselves are pinned in test_char_stencil.py)."""
    key = ("shell", n, steps)
    if key not in _cache:
        from curved_lbm import workloads
        from oracle.oracle import Oracle3D, available

        if not available():
            pytest.skip("oracle library not built")
        geom, mat, spec, kw = workloads.shell(n)
        o = Oracle3D(geom, material=mat, boundary=spec, threads=THREADS, char_stencil=stencil,
                     **kw)
        o.initialize_identity()
        o.run(steps)
        ref = {"f0": np.array(o.f0), "u_star": np.array(o.u_star)}
        o.refresh()
        ref["U"], ref["u"] = np.array(o.U), np.array(o.u)
        _cache[key] = ref
    return _cache[key]


def _gpu_shell(n, variant):
    from curved_lbm import workloads
    from curved_lbm.three_d import curved_boundary_warp3d as c3

    geom, mat, spec, kw = workloads.shell(n)
    s = c3.WarpSparseCurvedBoundaryLBM3D(geom, material=mat, boundary=spec, **kw)
    if variant is not None:
        s._select_variant(variant)
    s.initialize_identity()
    return s


def test_shell64_1000_steps_match_oracle():
    """A 64^3 spherical shell (90,240 active nodes) of the 3-D benchmark
    physics for 1000 steps with the default (autotuned) collide."""
    s = _gpu_shell(64, None)
    ref = _oracle_shell(64, 1000, s.characteristic_stencil)
    s.autotune(steps=10)
    s.run(1000)
    close_rel("f0", s.active_populations(), ref["f0"])
    close_rel("u_star", s.active_ustar(), ref["u_star"])
    s.refresh_current()
    close_rel("U", s.active_system_state(), ref["U"])
    close_rel("u", s.active_displacement(), ref["u"])
    _cache.pop(("shell", 64, 1000), None)


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
def test_shell_200_steps_match_oracle(variant):
    s = _gpu_shell(40, variant)
    ref = _oracle_shell(40, 200, s.characteristic_stencil)
    s.run(200)
    close_rel("f0", s.active_populations(), ref["f0"])
    close_rel("u_star", s.active_ustar(), ref["u_star"])
    s.refresh_current()
    close_rel("U", s.active_system_state(), ref["U"])
    close_rel("u", s.active_displacement(), ref["u"])


def test_shell96_gather_forms_bitwise_equal():
    """The 4-lanes-per-link characteristic gather (link-major tables) and the
    16-lane form (the reference's table layout): one state after 20 steps."""
    states = []
    for lm in (True, False):
        s = _gpu_shell(96, 0)
        if not lm:
            s._tables.pop("char_slot_lm")
            s._tables.pop("char_w_lm")
            s._problem = s._make_problem()
        s.run(20)
        states.append([s._host(t) for t in (s.f0, s.U, s.u, s.char_state)])
    for a, b in zip(*states):
        assert np.array_equal(a, b)


def test_shell96_collide_variants_bitwise_equal():
    """Every collide kernel, with and without the next step's moments
    overlapping the link kernels, eager and replayed from a graph: one state."""
    import torch

    want = None
    for v, overlap, graph in ((1, False, False), (0, False, False), (2, False, False),
                              (0, True, False), (0, True, True), (3, False, False),
                              (4, False, False), (3, False, True)):
        s = _gpu_shell(96, v)
        s.overlap_links = overlap
        if graph:
            g = s.capture_graph(10)
            for _ in range(3):
                g.launch()
            del g
        else:
            s.run(30)
        got = [s.active_populations(), s.active_ustar()]
        s.refresh_current()
        got += [s.active_system_state(), s.active_displacement()]
        assert np.isfinite(got[0]).all()
        if want is None:
            want = got
        else:
            for k, g, w in zip(("f0", "u_star", "U", "u"), got, want):
                np.testing.assert_array_equal(g, w, err_msg=f"{v} {overlap} {graph} {k}")
        del s
        torch.cuda.empty_cache()


def test_annulus512_fused_variants_bitwise_equal_per_phase():
    import torch

    base = _gpu_annulus(512, fused=False)
    base.run(30)
    want = [base.numpy_field(k) for k in ("f0", "u_star", "U", "u")]
    assert np.isfinite(want[0]).all()
    for v in range(11):
        s = _gpu_annulus(512, variant=v)
        s.run(30)
        for k, w in zip(("f0", "u_star", "U", "u"), want):
            np.testing.assert_array_equal(s.numpy_field(k), w, err_msg=f"variant {v} {k}")
        del s
        torch.cuda.empty_cache()


def test_annulus512_overlapped_links_bitwise_equal():
    """Inner tiles of the next step on a second stream while the link kernel
    runs: the same state as the serial step, every tile shape, eager and
    replayed from a graph."""
    import torch

    keys = ("f0", "u_star", "U", "u")
    for v in range(5):
        a = _gpu_annulus(512, variant=v)
        a.overlap_links = False
        a.run(30)
        want = [a.numpy_field(k) for k in keys]
        b = _gpu_annulus(512, variant=v)
        assert b.overlap_links and b._problem.n_tiles_inner > 0
        b.run(30)
        for k, w in zip(keys, want):
            np.testing.assert_array_equal(b.numpy_field(k), w, err_msg=f"variant {v} {k}")
        if v == 2:
            c = _gpu_annulus(512, variant=v)
            g = c.capture_graph(10)
            for _ in range(3):
                g.launch()
            for k, w in zip(keys, want):
                np.testing.assert_array_equal(c.numpy_field(k), w, err_msg=f"graph {k}")
            del g, c
        del a, b
        torch.cuda.empty_cache()


def test_annulus512_run_through_cached_graphs_equals_plain_run():
    """run() replays cached CUDA graphs for long even counts (recaptured when
    the buffers, settings or phase change); mixing graph and plain calls,
    odd counts and a variant switch gives the plain path's state."""
    a = _gpu_annulus(512)
    b = _gpu_annulus(512, graphs=True)
    for n in (40, 7, 40, 3, 16):
        a.run(n)
        b.run(n)
    b._select_variant(4)
    a._select_variant(4)
    a.run(24)
    b.run(24)
    assert len(b._graphs) >= 3 and a.steps == b.steps and a.time == b.time
    for k in ("f0", "u_star", "U", "u"):
        np.testing.assert_array_equal(a.numpy_field(k), b.numpy_field(k))


def test_annulus512_graph_equals_run():
    a = _gpu_annulus(512)
    b = _gpu_annulus(512)
    g = a.capture_graph(10)
    for _ in range(3):
        g.launch()
    b.run(30)
    assert a.time == b.time and a.steps == b.steps
    for k in ("f0", "u_star", "U", "u"):
        np.testing.assert_array_equal(a.numpy_field(k), b.numpy_field(k))
