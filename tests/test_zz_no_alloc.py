"""cvlbm2d_run_static_scratch: the allocation-free step, through the C-ABI.

It must give the same state as cvlbm2d_run (with a caller-owned link
scratch) over two calls in a row, an odd and an even step count, on the
benchmark traction annulus (fused node kernel, several hundred cut links).
Kept in its own file, named to be collected last, so that it runs both
alone and after every other GPU test in one process.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12
ATOL = 1e-15
FIELDS = ("f0", "u_star", "U", "u")


def _solver(n):
    from curved_lbm import workloads
    from curved_lbm.two_d import curved_boundary_warp as c2

    geom, mat, spec, kw = workloads.annulus(n)
    s = c2.WarpCurvedBoundaryLBM2D(geom, material=mat, boundary=spec, **kw)
    U, disp = workloads.annulus_initial_state(n)
    s.initialize_from_numpy(U=U, displacement=disp, init_order=2)
    return s


def _close(name, got, ref):
    """Element-wise |got - ref| <= ATOL + RTOL |ref|."""
    err = np.abs(got - ref)
    bad = err > ATOL + RTOL * np.abs(ref)
    assert not bad.any(), f"{name}: {int(bad.sum())} entries off, max abs err {float(err.max()):.3e}"


def test_static_scratch_matches_run_over_two_calls():
    import torch

    from curved_lbm import _native

    lib = _native.load()
    ref = _solver(160)
    s = _solver(160)
    assert 0 < s.geometry.n_links <= 16384
    assert s._problem.tiles, "the fused path must be the one exercised"

    ref.run(3)
    ref.run(4)

    fields = s._fields()
    fields.link_scratch = None  # ignored by the static entry point
    stream = _native.stream_ptr(s._tdev)
    t, step = float(s.time), int(s.steps)
    for nsteps in (3, 4):
        rc = lib.cvlbm2d_run_static_scratch(s._problem, fields, t, step, nsteps, stream)
        _native.check(rc, "cvlbm2d_run_static_scratch")
        for _ in range(nsteps):
            t += s.dt
        step += nsteps
    torch.cuda.synchronize(s._tdev)
    # the call hands back the f0/f1 exchange: 7 steps leave the state in f1
    assert fields.f0 == s.f1.data_ptr() and fields.f1 == s.f0.data_ptr()
    s.f0, s.f1 = s.f1, s.f0
    s.time, s.steps = t, step
    s._stress_current = False
    assert t == ref.time and step == ref.steps
    for k in FIELDS:
        _close(k, s.numpy_field(k), ref.numpy_field(k))


def test_static_scratch_calls_allocate_nothing():
    """After a first call (which looks up the array's address), further calls
    change neither the device's free memory nor the caching allocator."""
    import torch

    from curved_lbm import _native

    lib = _native.load()
    s = _solver(128)
    fields = s._fields()
    fields.link_scratch = None
    stream = _native.stream_ptr(s._tdev)

    def call(t, step, nsteps):
        rc = lib.cvlbm2d_run_static_scratch(s._problem, fields, t, step, nsteps, stream)
        _native.check(rc, "cvlbm2d_run_static_scratch")

    call(0.0, 0, 2)
    torch.cuda.synchronize(s._tdev)
    free0, _ = torch.cuda.mem_get_info(s._tdev)
    stats0 = torch.cuda.memory_stats(s._tdev)
    t, step = 2 * s.dt, 2
    for nsteps in (1, 2, 5):
        call(t, step, nsteps)
        t += nsteps * s.dt
        step += nsteps
    torch.cuda.synchronize(s._tdev)
    free1, _ = torch.cuda.mem_get_info(s._tdev)
    stats1 = torch.cuda.memory_stats(s._tdev)
    assert free1 == free0
    for key in ("allocation.all.allocated", "segment.all.allocated", "reserved_bytes.all.current"):
        assert stats1.get(key, 0) == stats0.get(key, 0), key


def test_static_scratch_rejects_too_many_links():
    from curved_lbm import _native

    lib = _native.load()
    s = _solver(64)
    big = _native.Problem2D.from_buffer_copy(s._problem)
    big.n_links = 16385
    rc = lib.cvlbm2d_run_static_scratch(ctypes.byref(big), s._fields(), 0.0, 0, 1,
                                        _native.stream_ptr(s._tdev))
    assert rc == -1
    msg = lib.cvlbm_last_error().decode()
    assert "16385" in msg and "16384" in msg
