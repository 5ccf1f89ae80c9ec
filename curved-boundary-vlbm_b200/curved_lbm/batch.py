"""Batched D2Q4x6 solves: many independent curved-boundary problems on one GPU.

``BatchedCurvedBoundaryLBM2D`` advances a list of ``WarpCurvedBoundaryLBM2D``
solvers (different geometries, load cases and lattice sizes) together: per
lattice step one persistent node launch and one persistent link launch cover
every instance (see ``cvlbm2d_batch_create`` in ``include/cvlbm.h``), the step
sequence is replayed from a CUDA graph, and each instance retires on its own
once its residual

    r = ||u - u_prev||_2 / (check_every * ||u||_2)   (sums over active nodes)

- the relative displacement change per step since the previous check - falls
below a tolerance after a minimum time (the end of its load ramp).  The
reference runs one solver object per geometry and has only an ``rms_v``
steady check in its case scripts; batching and this residual criterion are
additions.

Every instance follows exactly the arithmetic of its solo ``run``: a batched
instance's populations equal the solo solver's after the same number of
steps, bit for bit.
"""

from __future__ import annotations

import ctypes as C
import time as _time

import numpy as np

from . import _native


class BatchedCurvedBoundaryLBM2D:
    """Advance many ``WarpCurvedBoundaryLBM2D`` solvers together.

    The solvers must live on one CUDA device and support the fused step (one
    displacement sweep per step).  While the batch exists it owns their
    stepping: call :meth:`finish` before using a solver on its own again.
    """

    def __init__(self, solvers, *, tile_variant: int | None = None, grid_blocks: int = 0):
        if not solvers:
            raise ValueError("a batch needs at least one solver")
        self.solvers = list(solvers)
        dev = {s._tdev for s in self.solvers}
        if len(dev) != 1:
            raise ValueError("all batched solvers must be on the same device")
        self._tdev = dev.pop()
        for s in self.solvers:
            if not s._fused_possible:
                raise ValueError("a batched solver needs the fused-step tables")
            if s.local_displacement_sweeps > 1:
                raise ValueError("batched solvers take one displacement sweep per step")
        self._lib = _native.load()
        self.grid_blocks = int(grid_blocks)
        self.tile_variant = int(self.solvers[0].tile_variant if tile_variant is None
                                else tile_variant)
        self.handle = None
        self._graphs: dict = {}
        self._base_steps = None
        self._create()

    # -- native batch ----------------------------------------------------------
    def _create(self) -> None:
        n = len(self.solvers)
        for s in self.solvers:
            s._select_variant(self.tile_variant)
            s.invalid.zero_()
        probs = (_native.Problem2D * n)(*[s._problem for s in self.solvers])
        fields = (_native.Fields2D * n)(*[s._fields() for s in self.solvers])
        step0 = (C.c_int64 * n)(*[int(s.steps) for s in self.solvers])
        time0 = (C.c_double * n)(*[float(s.time) for s in self.solvers])
        h = C.c_void_p()
        _native.check(self._lib.cvlbm2d_batch_create(n, probs, fields, step0, time0,
                                                     self.tile_variant, self.grid_blocks,
                                                     C.byref(h)), "cvlbm2d_batch_create")
        self.handle = h
        self._base_steps = np.array([int(s.steps) for s in self.solvers], dtype=np.int64)

    def _destroy(self) -> None:
        for g in self._graphs.values():
            self._lib.cvlbm_graph_destroy(g)
        self._graphs = {}
        if self.handle:
            self._lib.cvlbm2d_batch_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass

    def _stream(self) -> int:
        return _native.stream_ptr(self._tdev)

    @property
    def n_instances(self) -> int:
        return len(self.solvers)

    def launch_grid(self) -> tuple[int, int]:
        """(persistent node grid size, number of (instance, tile) work items)."""
        g, w = C.c_int32(), C.c_int32()
        _native.check(self._lib.cvlbm2d_batch_launch_grid(self.handle, C.byref(g), C.byref(w)),
                      "cvlbm2d_batch_launch_grid")
        return int(g.value), int(w.value)

    # -- stepping ----------------------------------------------------------------
    def run(self, nsteps: int, *, check_every: int = 0, tol: float = 0.0,
            t_min: float = 0.0) -> None:
        """Advance every active instance by ``nsteps`` steps (asynchronous)."""
        if self.handle is None:
            raise RuntimeError("the batch was finished; build a new one")
        _native.check(self._lib.cvlbm2d_batch_run(self.handle, int(nsteps), int(check_every),
                                                  float(tol), float(t_min), self._stream()),
                      "cvlbm2d_batch_run")

    def graph(self, nsteps: int, *, check_every: int = 0, tol: float = 0.0,
              t_min: float = 0.0):
        """CUDA graph of ``run(nsteps, ...)``; returns a handle for :meth:`launch`."""
        key = (int(nsteps), int(check_every), float(tol), float(t_min))
        if key not in self._graphs:
            h = C.c_void_p()
            _native.check(self._lib.cvlbm2d_batch_graph_create(self.handle, *key, C.byref(h)),
                          "cvlbm2d_batch_graph_create")
            self._graphs[key] = h
        return self._graphs[key]

    def launch(self, graph) -> None:
        _native.check(self._lib.cvlbm_graph_launch(graph, self._stream()), "cvlbm_graph_launch")

    def status(self) -> dict:
        """Per-instance active flag, status, step index, time and last residual."""
        n = len(self.solvers)
        act = (C.c_int32 * n)()
        sta = (C.c_int32 * n)()
        steps = (C.c_int64 * n)()
        tim = (C.c_double * n)()
        res = (C.c_double * n)()
        _native.check(self._lib.cvlbm2d_batch_status(self.handle, act, sta, steps, tim, res,
                                                     self._stream()), "cvlbm2d_batch_status")
        return {"active": np.array(act[:], dtype=bool), "status": np.array(sta[:]),
                "steps": np.array(steps[:], dtype=np.int64), "time": np.array(tim[:]),
                "residual": np.array(res[:])}

    def run_to_residual(self, tol: float = 1.0e-8, *, check_every: int = 100,
                        t_min: float = 0.0, graph_steps: int = 1000,
                        max_steps: int = 10_000_000) -> dict:
        """Step until every instance has retired (converged or invalid).

        The step sequence runs from one CUDA graph of ``graph_steps`` steps
        with a residual check every ``check_every`` steps; the host reads the
        per-instance status between replays.  Returns the final status and
        the wall time.
        """
        import torch

        g = self.graph(graph_steps, check_every=check_every, tol=tol, t_min=t_min)
        torch.cuda.synchronize(self._tdev)
        t0 = _time.perf_counter()
        done = 0
        st = self.status()
        while st["active"].any() and done < max_steps:
            self.launch(g)
            done += graph_steps
            st = self.status()
        st["wall_s"] = _time.perf_counter() - t0
        st["batch_steps"] = done
        return st

    def autotune(self, steps: int = 20, variants=None) -> dict:
        """Time every compiled tile variant on this batch; keep the fastest.

        The populations and displacements are restored afterwards.  Returns
        {variant: ms per step}.
        """
        import torch

        saved = [(s.f0.clone(), s.f1.clone(), s.u_star.clone(), s.u_local_next.clone(),
                  s.U.clone(), s.u.clone(), s.time, s.steps) for s in self.solvers]
        cand = [v for v in (variants if variants is not None else range(5))
                if int(self._lib.cvlbm2d_tile_variant(int(v))) > 0]
        times = {}
        for v in cand:
            self._destroy()
            self.tile_variant = int(v)
            self._create()
            self.run(2)
            torch.cuda.synchronize(self._tdev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            self.run(steps)
            e1.record()
            e1.synchronize()
            times[v] = e0.elapsed_time(e1) / steps
            for s, sv in zip(self.solvers, saved):
                s.f0.copy_(sv[0]); s.f1.copy_(sv[1]); s.u_star.copy_(sv[2])
                s.u_local_next.copy_(sv[3]); s.U.copy_(sv[4]); s.u.copy_(sv[5])
                s.time, s.steps = sv[6], sv[7]
        best = min(times, key=times.get)
        self._destroy()
        self.tile_variant = best
        self._create()
        return times

    def finish(self, *, refresh: bool = True) -> dict:
        """Hand every instance's state back to its solver object.

        Updates time and step counters, exchanges f0/f1 and u*/u_next of the
        instances that took an odd number of batch steps, and (by default)
        refreshes U, u, P and sigma from the populations.
        """
        st = self.status()
        for k, s in enumerate(self.solvers):
            taken = int(st["steps"][k] - self._base_steps[k])
            if taken % 2 == 1:
                s.f0, s.f1 = s.f1, s.f0
                s.u_star, s.u_local_next = s.u_local_next, s.u_star
            s.steps = int(st["steps"][k])
            s.time = float(st["time"][k])
            s._stress_current = False
            if refresh:
                s.refresh_current()
        self._destroy()
        return st
