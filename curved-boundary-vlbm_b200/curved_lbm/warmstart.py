"""Learned warm start of the 3-D solver: a Fourier neural operator (FNO).

The surrogate maps a tube case (level set of the geometry and the end load:
stretch and twist) to the equilibrium displacement u and deformation
gradient F on the solver lattice, as a correction to the end kinematics
spread linearly along the tube (`kinematic_guess`).  The solver then starts from that state
(populations at equilibrium of U = (0, F), u* from u; the end displacement
applied at once) instead of the undeformed state with a load ramp, and the
plain damped relaxation converges from there; a prediction with a
non-positive Jacobian anywhere falls back to the cold start.  The reference
has no learned component; this module is an addition.

Network (channel-major activations x[b][c][g], g = lattice node):

    h0 = W0 x + b0                                  (lift, 8 -> 32 channels)
    h_{l+1} = act(W_l h_l + b_l + S_l(h_l)),  l = 0..3  (act = GELU, none last)
    y = Wp h_4 + bp                                 (project, 32 -> 12)
    S_l(h) = (h Phi) R_l Phi^T    (per retained mode k: 32 x 32 channel mix)

Phi is a truncated real Fourier basis on the lattice (cos / sin of the
lowest modes along each axis, orthonormal, padded with zero columns to a
multiple of 64).  The two spectral transforms of every layer, forward and
backward, run on the tensor cores (cvlbm_gemm_bf16: bf16 operands, fp32
accumulation); channel mixing, activations, the loss and Adam are this
library's CUDA-core kernels.  Weights are fp32.
"""

from __future__ import annotations

import math
import time as _time

import numpy as np

from . import _native

C_IN = 8
C_OUT = 12


def axis_basis(n: int, m: int) -> np.ndarray:
    """n x (2m-1) orthonormal real Fourier columns at cell centres."""
    x = (np.arange(n) + 0.5) / n
    cols = [np.full(n, 1.0 / math.sqrt(n))]
    for k in range(1, m):
        cols.append(math.sqrt(2.0 / n) * np.cos(2 * math.pi * k * x))
        cols.append(math.sqrt(2.0 / n) * np.sin(2 * math.pi * k * x))
    return np.stack(cols, axis=1)


def fourier_basis(shape, modes) -> np.ndarray:
    """G x M basis of the (nx, ny, nz) lattice (k fastest), M padded to 64."""
    bx, by, bz = (axis_basis(n, m) for n, m in zip(shape, modes))
    phi = np.einsum("ia,jb,kc->ijkabc", bx, by, bz).reshape(int(np.prod(shape)), -1)
    m = phi.shape[1]
    mp = -(-m // 64) * 64
    return np.pad(phi, ((0, 0), (0, mp - m)))


class FNO:
    """Fourier neural operator with native forward/backward (see module doc)."""

    def __init__(self, shape, *, modes=(4, 4, 8), width: int = 32, layers: int = 4,
                 batch: int = 4, device="cuda:0", seed: int = 0):
        import torch

        self.shape = tuple(int(s) for s in shape)
        self.G = int(np.prod(self.shape))
        if self.G % 64:
            raise ValueError("lattice node count must be a multiple of 64")
        if (batch * width) % 128:
            raise ValueError("batch * width must be a multiple of 128")
        self.C, self.L, self.B = int(width), int(layers), int(batch)
        self.dev = torch.device(device)
        self._lib = _native.load()
        phi = fourier_basis(self.shape, modes)
        self.M = phi.shape[1]
        bf = torch.bfloat16
        self.phi = torch.as_tensor(phi, dtype=torch.float32, device=self.dev).to(bf).contiguous()
        self.phiT = self.phi.t().contiguous()
        rng = np.random.default_rng(seed)
        C = self.C

        def w(o, i):
            return rng.normal(0.0, 1.0 / math.sqrt(i), (o, i))

        p = {"W0": w(C, C_IN), "b0": np.zeros(C)}
        for l in range(self.L):
            p[f"W{l + 1}"] = w(C, C)
            p[f"b{l + 1}"] = np.zeros(C)
            p[f"R{l + 1}"] = rng.normal(0.0, 1.0 / C, (self.M, C, C))
        p["Wp"] = w(C_OUT, C)
        p["bp"] = np.zeros(C_OUT)
        self.params = {k: torch.as_tensor(v, dtype=torch.float32, device=self.dev).contiguous()
                       for k, v in p.items()}
        self.grads = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self._adam = None
        self._err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        n_scr = max(int(self._lib.cvlbm_fno_pointwise_scratch(self.B, self.G, ci, co))
                    for ci, co in ((C_IN, C), (C, C), (C, C_OUT)))
        self._scratch = torch.empty(n_scr, dtype=torch.float32, device=self.dev)
        ws = max(int(self._lib.cvlbm_gemm_bf16_workspace(self.B * self.C, self.M, self.G)),
                 int(self._lib.cvlbm_gemm_bf16_workspace(self.B * self.C, self.G, self.M)))
        self._ws = torch.empty(ws // 4, dtype=torch.float32, device=self.dev)

    # -- native plumbing --------------------------------------------------------
    def _s(self):
        return _native.stream_ptr(self.dev)

    def _gemm(self, A, Bm, C, accumulate=0):
        M, K = A.shape
        N = Bm.shape[0]
        _native.check(self._lib.cvlbm_gemm_bf16(_native.ptr(A), _native.ptr(Bm), _native.ptr(C),
                                                M, N, K, A.stride(0), Bm.stride(0), C.stride(0),
                                                accumulate, _native.ptr(self._err),
                                                _native.ptr(self._ws), self._ws.numel() * 4,
                                                self._s()), "cvlbm_gemm_bf16")

    def _bf16(self, x):
        import torch

        out = torch.empty(x.shape, dtype=torch.bfloat16, device=self.dev)
        _native.check(self._lib.cvlbm_fno_to_bf16(x.numel(), _native.ptr(x), _native.ptr(out),
                                                  self._s()), "cvlbm_fno_to_bf16")
        return out

    def _pw(self, x, W, b, s=None, act=0, keep_z=False):
        import torch

        Cout, Cin = W.shape
        y = torch.empty((self.B, Cout, self.G), dtype=torch.float32, device=self.dev)
        z = torch.empty_like(y) if keep_z else None
        _native.check(self._lib.cvlbm_fno_pointwise_fwd(
            self.B, self.G, Cin, Cout, _native.ptr(x), _native.ptr(W), _native.ptr(b),
            _native.ptr(s), act, _native.ptr(z), _native.ptr(y), self._s()),
            "cvlbm_fno_pointwise_fwd")
        return y, z

    def _pw_bwd(self, dz, x, W, dW, db, dx=None, accumulate=0):
        Cout, Cin = W.shape
        _native.check(self._lib.cvlbm_fno_pointwise_bwd(
            self.B, self.G, Cin, Cout, _native.ptr(dz), _native.ptr(x), _native.ptr(W),
            _native.ptr(dx), accumulate, _native.ptr(dW), _native.ptr(db),
            _native.ptr(self._scratch), self._s()), "cvlbm_fno_pointwise_bwd")

    # -- forward / backward ------------------------------------------------------
    def forward(self, x):
        """x: [B, 8, G] fp32 -> y: [B, 12, G]; keeps what backward needs."""
        import torch

        P, B, C, G, M = self.params, self.B, self.C, self.G, self.M
        cache = {"x": x}
        h, _ = self._pw(x, P["W0"], P["b0"])
        for l in range(1, self.L + 1):
            hb = self._bf16(h).view(B * C, G)
            a = torch.empty((B * C, M), dtype=torch.float32, device=self.dev)
            self._gemm(hb, self.phiT, a)  # a = h Phi
            bh = torch.empty((B * C, M), dtype=torch.bfloat16, device=self.dev)
            _native.check(self._lib.cvlbm_fno_spec_mix_fwd(B, C, M, _native.ptr(a),
                                                           _native.ptr(P[f"R{l}"]),
                                                           _native.ptr(bh), self._s()),
                          "cvlbm_fno_spec_mix_fwd")
            s = torch.empty((B * C, G), dtype=torch.float32, device=self.dev)
            self._gemm(bh, self.phi, s)  # s = bh Phi^T
            act = 1 if l < self.L else 0
            hn, z = self._pw(h, P[f"W{l}"], P[f"b{l}"], s=s, act=act, keep_z=True)
            cache[l] = (h, a, z)
            h = hn
        cache["h"] = h
        y, _ = self._pw(h, P["Wp"], P["bp"])
        self._cache = cache
        return y

    def backward(self, dy):
        """Gradients of all parameters from dL/dy (into self.grads)."""
        import torch

        P, Gr, B, C, G, M = self.params, self.grads, self.B, self.C, self.G, self.M
        cache = self._cache
        dh = torch.empty((B, C, G), dtype=torch.float32, device=self.dev)
        self._pw_bwd(dy, cache["h"], P["Wp"], Gr["Wp"], Gr["bp"], dx=dh)
        for l in range(self.L, 0, -1):
            h, a, z = cache[l]
            if l < self.L:
                dz = torch.empty_like(dh)
                _native.check(self._lib.cvlbm_fno_gelu_bwd(dh.numel(), _native.ptr(z),
                                                           _native.ptr(dh), _native.ptr(dz),
                                                           self._s()), "cvlbm_fno_gelu_bwd")
            else:
                dz = dh
            dprev = torch.empty((B, C, G), dtype=torch.float32, device=self.dev)
            self._pw_bwd(dz, h, P[f"W{l}"], Gr[f"W{l}"], Gr[f"b{l}"], dx=dprev)
            dzb = self._bf16(dz).view(B * C, G)
            dbh = torch.empty((B * C, M), dtype=torch.float32, device=self.dev)
            self._gemm(dzb, self.phiT, dbh)  # dbh = dz Phi
            da = torch.empty((B * C, M), dtype=torch.bfloat16, device=self.dev)
            _native.check(self._lib.cvlbm_fno_spec_mix_bwd(
                B, C, M, _native.ptr(a), _native.ptr(dbh), _native.ptr(P[f"R{l}"]),
                _native.ptr(da), _native.ptr(Gr[f"R{l}"]), self._s()), "cvlbm_fno_spec_mix_bwd")
            self._gemm(da, self.phi, dprev.view(B * C, G), accumulate=1)  # += da Phi^T
            dh = dprev
        self._pw_bwd(dh, cache["x"], P["W0"], Gr["W0"], Gr["b0"])
        return Gr

    def loss_grad(self, y, t, mask, wch):
        """Masked weighted MSE and dL/dy (native)."""
        import torch

        n_parts = 256
        dy = torch.empty_like(y)
        part = torch.empty(n_parts, dtype=torch.float32, device=self.dev)
        cnt = float(mask.sum().item()) * C_OUT
        _native.check(self._lib.cvlbm_fno_mse(self.B, C_OUT, self.G, _native.ptr(y),
                                              _native.ptr(t), _native.ptr(mask),
                                              _native.ptr(wch), 1.0 / max(cnt, 1.0),
                                              _native.ptr(dy), _native.ptr(part), n_parts,
                                              self._s()), "cvlbm_fno_mse")
        return part, dy

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        import torch

        if self._adam is None:
            self._adam = {"t": 0, "m": {k: torch.zeros_like(v) for k, v in self.params.items()},
                          "v": {k: torch.zeros_like(v) for k, v in self.params.items()}}
        st = self._adam
        st["t"] += 1
        lr_t = lr * math.sqrt(1 - b2 ** st["t"]) / (1 - b1 ** st["t"])
        for k, p in self.params.items():
            _native.check(self._lib.cvlbm_fno_adam(p.numel(), _native.ptr(p),
                                                   _native.ptr(self.grads[k]),
                                                   _native.ptr(st["m"][k]),
                                                   _native.ptr(st["v"][k]), lr_t, b1, b2, eps,
                                                   self._s()), "cvlbm_fno_adam")

    def gemm_ok(self) -> bool:
        return int(self._err.item()) == 0


# ---------------------------------------------------------------------------
# Tube data: features, solver equilibria, warm and cold starts
# ---------------------------------------------------------------------------
def _tube_grid(prm: dict, nxy: int):
    from . import workloads

    nx, ny, nz, dx = workloads.tube_lattice(nxy)
    cx, cy = 0.5 * nx * dx, 0.5 * ny * dx
    z0 = 0.5 * (nz * dx - workloads.TUBE_LENGTH)
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    z = (np.arange(nz) + 0.5) * dx
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    zeta = np.clip((Z - z0) / workloads.TUBE_LENGTH, 0.0, 1.0)
    return X, Y, Z, cx, cy, z0, zeta, dx


def kinematic_guess(prm: dict, nxy: int) -> np.ndarray:
    """[12, G] (u, F - I) of the end kinematics spread linearly along the tube:
    at axial fraction zeta the section is stretched by zeta (stretch - 1) L and
    turned by zeta * twist - exactly the clamped left end and the prescribed
    right end, with no radial (Poisson) or end-layer correction.  The
    surrogate learns the correction to this field."""
    from . import workloads

    X, Y, Z, cx, cy, z0, zeta, dx = _tube_grid(prm, nxy)
    th = zeta * prm["twist"]
    c, s = np.cos(th), np.sin(th)
    ux = (c - 1.0) * (X - cx) - s * (Y - cy)
    uy = s * (X - cx) + (c - 1.0) * (Y - cy)
    uz = zeta * (prm["stretch"] - 1.0) * workloads.TUBE_LENGTH
    u = np.stack([ux, uy, uz])
    F = np.zeros((9,) + X.shape)
    for r in range(3):
        g = np.gradient(u[r], dx, axis=(0, 1, 2))
        for col in range(3):
            F[3 * r + col] = g[col]
    return np.concatenate([u, F]).reshape(12, -1)


def tube_features(prm: dict, nxy: int) -> tuple[np.ndarray, np.ndarray]:
    """([8, G] input channels, [G] material mask) of one tube case: mask, level
    set, coordinates and the kinematic guess of u."""
    from . import workloads

    X, Y, Z, cx, cy, z0, zeta, dx = _tube_grid(prm, nxy)
    r = np.sqrt((X - cx) ** 2 + (Y - cy) ** 2)
    phi = np.maximum.reduce((r - prm["r_out"], prm["r_in"] - r, z0 - Z,
                             Z - z0 - workloads.TUBE_LENGTH))
    mask = (phi <= 0.0).astype(np.float32)
    g = kinematic_guess(prm, nxy)[:3].reshape((3,) + X.shape)
    f = np.stack([mask, np.clip(phi / 0.3, -1, 1), (X - cx) / 0.9, (Y - cy) / 0.9,
                  2 * zeta - 1, g[0] / 0.3, g[1] / 0.3, g[2] / 0.6])
    return f.reshape(C_IN, -1).astype(np.float32), mask.reshape(-1)


def solver_targets(solver) -> np.ndarray:
    """[12, G]: u (3) and F - I (9) on the lattice, zero outside the material."""
    ai, aj, ak = solver.active_i, solver.active_j, solver.active_k
    nx, ny, nz = solver.nx, solver.ny, solver.nz
    u = solver.active_displacement()
    U = solver.active_system_state()
    F = U[3:12].copy()
    F[0] -= 1.0
    F[4] -= 1.0
    F[8] -= 1.0
    out = np.zeros((12, nx, ny, nz))
    out[:3, ai, aj, ak] = u
    out[3:, ai, aj, ak] = F
    return out.reshape(12, -1)


def make_tube_solver(prm: dict, nxy: int, *, ramp_time: float, device="cuda:0"):
    from . import workloads
    from .three_d import curved_boundary_warp3d as c3

    g = workloads.tube_geometry(prm, nxy)
    mat, spec, kw = workloads.tube_case(prm, nxy, ramp_time=ramp_time)
    return c3.WarpSparseCurvedBoundaryLBM3D(g, material=mat, boundary=spec, device=device, **kw)


def run_to_residual(solver, tol: float, *, check: int = 100, t_min: float = 0.0,
                    max_steps: int = 400_000, graph=None, consecutive: int = 1) -> dict:
    """Step until |u - u_prev|_2 / (check |u|_2) < tol (relative displacement
    change per step over a check interval) at `consecutive` checks in a row,
    after t >= t_min.  (More than one check keeps a lightly damped
    oscillation from passing the test at a turning point.)"""
    import torch

    g = graph if graph is not None else solver.capture_graph(check)
    prev = solver.u.clone()
    torch.cuda.synchronize()
    t0 = _time.perf_counter()
    steps0 = solver.steps
    r = float("inf")
    run = 0
    while solver.steps - steps0 < max_steps:
        g.launch()
        du = torch.linalg.vector_norm(solver.u - prev).item()
        nu = torch.linalg.vector_norm(solver.u).item()
        r = du / (check * nu) if nu > 0 else float("inf")
        prev.copy_(solver.u)
        run = run + 1 if (solver.time >= t_min and r < tol) else 0
        if run >= consecutive:
            break
    torch.cuda.synchronize()
    return {"wall_s": _time.perf_counter() - t0, "steps": solver.steps - steps0, "residual": r,
            "invalid": bool(solver.invalid_state())}


def run_batch_to_residual(solvers: list, tol: float, *, check: int = 100, t_min=0.0,
                          max_steps=400_000, consecutive: int = 1) -> dict:
    """`run_to_residual` for several independent solvers at once.

    Each solver replays its own captured `check`-step graph on its own CUDA
    stream, so the small per-solver launches of one round run side by side
    on the SMs; the residual norms of every solver land in one device array
    read back with a single copy per round.  A solver stops at the first
    round its residual criterion holds, exactly as it would alone (same
    graph, same steps), so each solver's steps and final state equal those of
    a solo `run_to_residual`.  `t_min` and `max_steps` are one value for
    all or one per solver.  Returns per-solver steps / residual / invalid and the wall time
    of the whole batch."""
    import torch

    if not solvers:
        return {"wall_s": 0.0, "solvers": []}
    dev = solvers[0]._tdev
    if any(s._tdev != dev for s in solvers):
        raise ValueError("run_batch_to_residual: every solver must live on the same device")
    n = len(solvers)
    t_mins = [float(t) for t in t_min] if isinstance(t_min, (list, tuple)) else [float(t_min)] * n
    caps = [int(v) for v in max_steps] if isinstance(max_steps, (list, tuple)) else [int(max_steps)] * n
    if len(t_mins) != n or len(caps) != n:
        raise ValueError("run_batch_to_residual: one t_min / max_steps per solver")
    graphs = [s.capture_graph(check) for s in solvers]
    streams = [torch.cuda.Stream(device=dev) for _ in range(n)]
    prev = [s.u.clone() for s in solvers]
    norms = torch.zeros((n, 2), dtype=torch.float64, device=dev)
    steps0 = [s.steps for s in solvers]
    res = [float("inf")] * n
    runs = [0] * n
    active = list(range(n))
    torch.cuda.synchronize(dev)
    main = torch.cuda.current_stream(dev)
    for st in streams:
        st.wait_stream(main)
    t0 = _time.perf_counter()
    while active:
        for i in active:
            s = solvers[i]
            with torch.cuda.stream(streams[i]):
                graphs[i].launch()
                torch.linalg.vector_norm(s.u - prev[i], out=norms[i, 0])
                torch.linalg.vector_norm(s.u, out=norms[i, 1])
                prev[i].copy_(s.u)
        for i in active:
            main.wait_stream(streams[i])
        h = norms.cpu().numpy()
        still = []
        for i in active:
            s = solvers[i]
            du, nu = float(h[i, 0]), float(h[i, 1])
            res[i] = du / (check * nu) if nu > 0 else float("inf")
            runs[i] = runs[i] + 1 if (s.time >= t_mins[i] and res[i] < tol) else 0
            if runs[i] < consecutive and s.steps - steps0[i] < caps[i]:
                still.append(i)
        active = still
        for i in active:
            streams[i].wait_stream(main)
    torch.cuda.synchronize(dev)
    wall = _time.perf_counter() - t0
    return {"wall_s": wall,
            "solvers": [{"steps": s.steps - s0, "residual": r, "invalid": bool(s.invalid_state())}
                        for s, s0, r in zip(solvers, steps0, res)]}


def warm_initialize(solver, pred: np.ndarray) -> bool:
    """Start `solver` from a predicted [12, G] (u, F - I) field; returns False
    (and leaves the solver undeformed) if the prediction has det F <= floor
    at some active node."""
    nx, ny, nz = solver.nx, solver.ny, solver.nz
    p = pred.reshape(12, nx, ny, nz)[:, solver.active_i, solver.active_j, solver.active_k]
    F = p[3:12].copy()
    F[0] += 1.0
    F[4] += 1.0
    F[8] += 1.0
    Fm = F.reshape(3, 3, -1)
    det = (Fm[0, 0] * (Fm[1, 1] * Fm[2, 2] - Fm[1, 2] * Fm[2, 1])
           - Fm[0, 1] * (Fm[1, 0] * Fm[2, 2] - Fm[1, 2] * Fm[2, 0])
           + Fm[0, 2] * (Fm[1, 0] * Fm[2, 1] - Fm[1, 1] * Fm[2, 0]))
    if not np.all(det > 10.0 * solver.jacobian_floor):
        return False
    U = np.zeros((12, solver.n_active))
    U[3:] = F
    solver._initialize_from_active(U, p[:3], init_order=1)
    return True


def generate_equilibria(params: list[dict], nxy: int, tol: float, device="cuda:0",
                        check: int = 100, batch: int = 32) -> list[dict]:
    """Cold-start solves of the given tube cases to the residual tolerance:
    the solver's own equilibria, the surrogate's training data.  `batch`
    solvers at a time run side by side (`run_batch_to_residual`)."""
    from . import workloads

    out = []
    for k in range(0, len(params), max(1, batch)):
        group = params[k:k + max(1, batch)]
        solvers = [make_tube_solver(prm, nxy, ramp_time=workloads.TUBE_RAMP_TIME, device=device)
                   for prm in group]
        info = run_batch_to_residual(solvers, tol, check=check, t_min=workloads.TUBE_RAMP_TIME)
        for prm, s, si in zip(group, solvers, info["solvers"]):
            x, mask = tube_features(prm, nxy)
            out.append({"params": prm, "x": x, "mask": mask,
                        "target": solver_targets(s) - kinematic_guess(prm, nxy) * mask[None, :],
                        "steps": si["steps"], "wall_s": info["wall_s"] / len(group),
                        "residual": si["residual"], "invalid": si["invalid"]})
        del solvers
    return out


def output_scale(t_all: np.ndarray, m_all: np.ndarray, device="cpu") -> np.ndarray:
    """Per-channel RMS of the masked training targets [n, C_OUT, G] over the
    training set of every rank (each rank passes its own share)."""
    import torch

    from . import replicas

    w = m_all[:, None, :]
    num = torch.as_tensor((t_all ** 2 * w).sum(axis=(0, 2)), dtype=torch.float64, device=device)
    den = torch.as_tensor(np.broadcast_to(w.sum(axis=(0, 2)), num.shape).copy(),
                          dtype=torch.float64, device=device)
    replicas.allreduce_([num, den])
    std = np.sqrt(num.cpu().numpy() / np.maximum(den.cpu().numpy(), 1))
    return np.maximum(std, 1e-6).astype(np.float32)


class Surrogate:
    """FNO plus the per-channel output scaling of the training set.

    Under an open process group `fit` trains data-parallel: every rank holds
    its own share of the equilibria, draws the same number of batches per
    epoch, and the gradients are averaged over the ranks (one flat
    all-reduce) before each Adam step, so every rank keeps the same weights.
    """

    def __init__(self, nxy: int, *, modes=(4, 4, 8), batch: int = 4, device="cuda:0",
                 seed: int = 0):
        from . import workloads

        nx, ny, nz, _ = workloads.tube_lattice(nxy)
        self.nxy = nxy
        self.net = FNO((nx, ny, nz), modes=modes, batch=batch, device=device, seed=seed)
        self.scale = np.ones(C_OUT, dtype=np.float32)
        self.history: list[float] = []

    def _batches(self, data, rng, n: int | None = None):
        """Shuffled batches of B cases, padded by resampling to n cases (at
        least len(data)) and to a multiple of B."""
        B = self.net.B
        idx = rng.permutation(len(data))
        n = max(len(data), n or 0)
        n = -(-n // B) * B
        if len(idx) < n:
            idx = np.concatenate([idx, rng.choice(len(data), n - len(idx))])
        return idx.reshape(-1, B)

    def fit(self, data, *, epochs: int = 100, lr: float = 2e-3, seed: int = 0) -> list[float]:
        import torch

        from . import replicas

        net = self.net
        dev = net.dev
        world, rank = replicas.world_and_rank()
        if not data:
            raise ValueError("Surrogate.fit needs at least one training case on every rank")
        t_all = np.stack([d["target"] for d in data])
        m_all = np.stack([d["mask"] for d in data])
        self.scale = output_scale(t_all, m_all, dev)
        X = torch.as_tensor(np.stack([d["x"] for d in data]), device=dev)
        T = torch.as_tensor((t_all / self.scale[None, :, None]).astype(np.float32), device=dev)
        Mk = torch.as_tensor(m_all.astype(np.float32), device=dev)
        wch = torch.ones(C_OUT, dtype=torch.float32, device=dev)
        rng = np.random.default_rng(seed + 1000 * rank)
        n_max = torch.tensor([float(len(data))], dtype=torch.float64, device=dev)
        replicas.allreduce_([n_max], op="max")  # equal batch counts on every rank
        n_max = int(n_max.item())
        grads = list(net.grads.values())
        hist = []
        for ep in range(epochs):
            lr_e = lr * 0.5 * (1 + math.cos(math.pi * ep / epochs))
            tot = torch.zeros(1, dtype=torch.float64, device=dev)
            batches = self._batches(data, rng, n_max)
            for b in batches:
                bi = torch.as_tensor(b, device=dev)
                y = net.forward(X[bi].contiguous())
                part, dy = net.loss_grad(y, T[bi].contiguous(), Mk[bi].contiguous(), wch)
                net.backward(dy)
                if world > 1:
                    replicas.allreduce_(grads)
                    for g in grads:
                        g.mul_(1.0 / world)
                net.adam_step(lr=lr_e)
                tot += part.sum().double()
            replicas.allreduce_([tot])
            hist.append(float(tot.item()) / (len(batches) * world))
        if not net.gemm_ok():
            raise RuntimeError("tensor-core GEMM reported incomplete MMAs during training")
        self.history = hist
        return hist

    def predict(self, feats: list[np.ndarray]) -> list[np.ndarray]:
        import torch

        net = self.net
        out = []
        for k in range(0, len(feats), net.B):
            chunk = feats[k:k + net.B]
            pad = chunk + [chunk[-1]] * (net.B - len(chunk))
            y = net.forward(torch.as_tensor(np.stack(pad), device=net.dev))
            y = y.double().cpu().numpy() * self.scale[None, :, None]
            out.extend(list(y[:len(chunk)]))
        return out


def _rel_err(a: np.ndarray, b: np.ndarray, mask: np.ndarray) -> float:
    m = mask.astype(bool)
    return float(np.linalg.norm((a - b)[:, m]) / max(np.linalg.norm(b[:, m]), 1e-300))


def _solver_state(s) -> np.ndarray:
    import torch

    torch.cuda.synchronize(s._tdev)
    return torch.cat([s.u.reshape(-1), s.U.reshape(-1), s.f0.reshape(-1)]).cpu().numpy()


def train_and_compare(*, nxy: int = 32, n_train: int = 64, n_test: int = 4, epochs: int = 200,
                      tol: float = 1e-8, seed: int = 7, device="cuda:0", modes=(4, 4, 8),
                      lr: float = 2e-3, gen_batch: int = 32, consecutive: int = 1) -> dict:
    """Generate solver equilibria, train the surrogate, then compare warm and
    cold starts on held-out cases.

    Per held-out case: the cold start (undeformed, end load ramped over
    TUBE_RAMP_TIME) and the warm start (surrogate prediction, end load at
    once) both run to `tol`; the cold run then continues to tol/100, whose
    field is the converged reference both final errors are measured against.

    Wall times: cold and warm plain (one solve after another, the way the
    reference runs its cases) and batched (every held-out case side by side,
    `run_batch_to_residual`).  The batched runs are checked to reach the
    plain runs' step counts and states bit for bit.  At equal final error:
    the warm solves stopped at the first check where their error against the
    converged field is at or below the cold run's final error, timed batched
    (`speedup_batched_equal_error`).
    """
    from . import replicas, workloads

    world, rank = replicas.world_and_rank()
    if n_train < world:
        # every rank must hold training cases: a rank with none would fail
        # before its first gradient all-reduce and leave the others waiting
        raise ValueError(f"n_train={n_train} is smaller than the number of ranks ({world})")
    dx = workloads.tube_lattice(nxy)[3]
    params = workloads.tube_params(n_train + n_test, seed, min_wall=4.0 * dx)
    t0 = _time.perf_counter()
    # under a process group every rank solves its own share of the cases
    train = generate_equilibria(replicas.deal(params[:n_train], rank, world), nxy, tol, device,
                                batch=gen_batch)
    gen_s = _time.perf_counter() - t0
    sur = Surrogate(nxy, modes=modes, device=device, seed=seed)
    t0 = _time.perf_counter()
    hist = sur.fit(train, epochs=epochs, lr=lr, seed=seed)
    fit_s = _time.perf_counter() - t0
    (gen_s, fit_s), (steps_sum, n_done) = replicas.reduce_times_and_counts(
        [gen_s, fit_s], [sum(d["steps"] for d in train), len(train)], device=device)
    if rank != 0:  # the held-out comparison runs on one GPU
        return {"rank": rank, "n_train_local": len(train)}
    ramp = workloads.TUBE_RAMP_TIME
    test = params[n_train:]
    feats = [tube_features(prm, nxy) for prm in test]
    preds = [p + kinematic_guess(prm, nxy) * m[None, :]
             for prm, p, (_, m) in zip(test, sur.predict([x for x, _ in feats]), feats)]

    def warm_solver(prm, pred):
        s = make_tube_solver(prm, nxy, ramp_time=0.0, device=device)
        if warm_initialize(s, pred):
            return s, True, 0.0
        # fallback: the plain cold start
        return make_tube_solver(prm, nxy, ramp_time=ramp, device=device), False, ramp

    cases = []
    for prm, pred, (x, mask) in zip(test, preds, feats):
        cold = make_tube_solver(prm, nxy, ramp_time=ramp, device=device)
        ci = run_to_residual(cold, tol, t_min=ramp, consecutive=consecutive)
        u_cold = solver_targets(cold)
        st_cold = _solver_state(cold)
        run_to_residual(cold, tol / 100.0)
        ref = solver_targets(cold)
        warm, ok, t_min = warm_solver(prm, pred)
        wi = run_to_residual(warm, tol, t_min=t_min, consecutive=consecutive)
        u_warm = solver_targets(warm)
        cases.append({"params": prm, "warm_ok": ok, "cold_steps": ci["steps"],
                      "warm_steps": wi["steps"], "cold_wall_s": ci["wall_s"],
                      "warm_wall_s": wi["wall_s"], "cold_err": _rel_err(u_cold, ref, mask),
                      "warm_err": _rel_err(u_warm, ref, mask),
                      "prediction_err": _rel_err(pred, ref, mask),
                      "guess_err": _rel_err(kinematic_guess(prm, nxy) * mask[None, :], ref, mask),
                      "warm_invalid": wi["invalid"], "cold_invalid": ci["invalid"],
                      "_cold_state": st_cold, "_warm_state": _solver_state(warm), "_ref": ref})
        del cold, warm
    # the same solves again, every case side by side
    colds = [make_tube_solver(prm, nxy, ramp_time=ramp, device=device) for prm in test]
    cb = run_batch_to_residual(colds, tol, t_min=ramp, consecutive=consecutive)
    cold_same = all(c["cold_steps"] == b["steps"] and np.array_equal(c["_cold_state"],
                                                                      _solver_state(s))
                    for c, b, s in zip(cases, cb["solvers"], colds))
    del colds
    built = [warm_solver(prm, pred) for prm, pred in zip(test, preds)]
    wb = run_batch_to_residual([s for s, _, _ in built], tol, t_min=[t for _, _, t in built],
                               consecutive=consecutive)
    warm_same = all(c["warm_steps"] == b["steps"] and np.array_equal(c["_warm_state"],
                                                                      _solver_state(s))
                    for c, b, (s, _, _) in zip(cases, wb["solvers"], built))
    del built
    # equal final error: the first check (every `check` steps) at which the
    # warm run's error against the converged field is at or below the cold
    # run's final error (calibration pass, untimed), then the warm solves
    # timed side by side to exactly those step counts
    check = 100
    eq_steps = []
    for prm, pred, (x, mask), c in zip(test, preds, feats, cases):
        warm, ok, t_min = warm_solver(prm, pred)
        g = warm.capture_graph(check)
        steps = None
        while warm.steps < 50 * max(c["cold_steps"], check):
            g.launch()
            if _rel_err(solver_targets(warm), c["_ref"], mask) <= c["cold_err"]:
                steps = warm.steps
                break
        c["warm_steps_equal_error"] = steps
        eq_steps.append(steps if steps is not None else warm.steps)
        del g, warm
    built = [warm_solver(prm, pred) for prm, pred in zip(test, preds)]
    we = run_batch_to_residual([s for s, _, _ in built], 0.0, check=check, max_steps=eq_steps)
    eq_errs = [_rel_err(solver_targets(s), c["_ref"], m) for (s, _, _), c, (_, m)
               in zip(built, cases, feats)]
    for c, e in zip(cases, eq_errs):
        c["warm_err_equal_error"] = e
    del built
    for c in cases:
        del c["_cold_state"], c["_warm_state"], c["_ref"]
    cold_w = sum(c["cold_wall_s"] for c in cases)
    warm_w = sum(c["warm_wall_s"] for c in cases)
    return {"nxy": nxy, "dx": dx, "min_wall": 4.0 * dx, "n_train": n_train, "n_test": n_test,
            "epochs": epochs, "tol": tol, "consecutive_checks": consecutive,
            "modes": list(modes), "generate_s": gen_s,
            "fit_s": fit_s, "train_loss_first": hist[0], "train_loss_last": hist[-1],
            "train_steps_mean": steps_sum / max(n_done, 1), "ranks": world,
            "cases": cases, "cold_wall_s": cold_w, "warm_wall_s": warm_w,
            "cold_batched_wall_s": cb["wall_s"], "warm_batched_wall_s": wb["wall_s"],
            "batched_equals_plain": bool(cold_same and warm_same),
            "warm_batched_equal_error_wall_s": we["wall_s"],
            "equal_error_reached": all(c["warm_steps_equal_error"] is not None for c in cases),
            "speedup_batched_equal_error": cold_w / max(we["wall_s"], 1e-12),
            "speedup_steps_equal_error": sum(c["cold_steps"] for c in cases)
            / max(sum(eq_steps), 1),
            "speedup_wall": cold_w / max(warm_w, 1e-12),
            "speedup_batched": cold_w / max(wb["wall_s"], 1e-12),
            "speedup_steps": sum(c["cold_steps"] for c in cases)
            / max(sum(c["warm_steps"] for c in cases), 1)}
