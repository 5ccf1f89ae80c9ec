"""Python driver of the CPU oracle -- TEST INFRASTRUCTURE.

Mirrors the reference solver classes closely enough to replay a case:
configuration processing, host initialisation (the NumPy restatements of the
reference's init functions), the in-place boundary pass and the time step,
all evaluated by ``libcvlbm_oracle.so`` (``oracle/cvlbm_oracle.c``) on host
arrays.  Used only by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_lib = None


def available() -> bool:
    try:
        load()
        return True
    except Exception:
        return False


def load():
    global _lib
    if _lib is None:
        path = _build.build()
        _lib = C.CDLL(str(path))
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class _Scratch2(C.Structure):
    _fields_ = [("bc_diag", C.c_void_p), ("bc_rhs", C.c_void_p)]


class Oracle2D:
    """Serial/OpenMP CPU replay of WarpCurvedBoundaryLBM2D (reference C2:3618-4472)."""

    def __init__(self, geometry, *, material, boundary, lattice_speed=5.0, collision_omega=2.0,
                 boundary_reconstruction="bfl", jacobian_floor=1e-12, source_mode="none",
                 source_vector=(0.0,) * 6, damping_gamma=0.0, local_compatibility_interval=0,
                 local_compatibility_blend=0.05, local_compatibility_interior_only=True,
                 local_displacement_interval=0, local_displacement_sweeps=1,
                 local_displacement_relax=0.85, local_displacement_boundary_weight=20.0,
                 local_displacement_boundary_id=2, normal_jacobian=None, neumann_solver=None,
                 collision_model="bgk", ghost_omega=None, kinetic_filter_strength=0.0,
                 threads=1, **_unused):
        from curved_lbm import _native
        from curved_lbm.two_d import curved_boundary_warp as c2
        from curved_lbm.two_d import vector_nonlinear_elastic_warp as v2

        self.lib = load()
        self.g = g = geometry
        self.nx, self.ny = g.nx, g.ny
        self.N = N = g.nx * g.ny
        self.dx, self.dy = g.dx, g.dy
        self.dt = g.dx / float(lattice_speed)
        self.c = float(lattice_speed)
        self.material = material
        self.threads = int(threads)
        self.source_mode = v2.source_id(source_mode)
        sp = np.zeros(6)
        if self.source_mode == v2.SOURCE_CONSTANT:
            sp[: len(source_vector)] = np.asarray(source_vector, float)[:6]
        elif self.source_mode == v2.SOURCE_DAMPING:
            sp[0] = float(damping_gamma)
        self.source_params = sp
        nsolver = c2.neumann_solver_name(neumann_solver, material)
        nj = c2.normal_jacobian_id(normal_jacobian)
        kind, mode, params = boundary.tables(c2.MAX_BOUNDARY_IDS)
        self._keep = []

        def keep(a, dtype):
            a = np.ascontiguousarray(a, dtype=dtype)
            self._keep.append(a)
            return a

        p = _native.Problem2D()
        p.nx, p.ny, p.n_links = g.nx, g.ny, g.n_links
        p.recon = c2.boundary_reconstruction_id(boundary_reconstruction)
        p.normal_solver = 2 if nsolver == "energy" else nj
        p.source_mode = self.source_mode
        p.dx, p.dy, p.dt, p.omega, p.c = g.dx, g.dy, self.dt, float(collision_omega), self.c
        for i in range(6):
            p.source[i] = sp[i]
        p.mat = _native.Material(material.id, 0, material.lam, material.mu, material.param0,
                                 material.param1, material.param2, float(jacobian_floor))
        p.disp_interval = int(max(0, local_displacement_interval))
        p.disp_sweeps = int(local_displacement_sweeps)
        p.disp_bid = int(local_displacement_boundary_id)
        p.rep_interval = int(max(0, local_compatibility_interval))
        p.interior_only = int(bool(local_compatibility_interior_only))
        p.relax = float(local_displacement_relax)
        p.weight = float(local_displacement_boundary_weight)
        p.blend = float(local_compatibility_blend)
        p.collision_model = 1 if collision_model == "mrt_ghost" else 0
        p.ghost_omega = float(collision_omega if ghost_omega is None else ghost_omega)
        p.kinetic_filter = float(kinetic_filter_strength)
        i32, f64 = np.int32, np.float64
        p.active = _ptr(keep(g.active.reshape(-1), i32))
        for name in ("link_i", "link_j", "link_q"):
            setattr(p, name, _ptr(keep(getattr(g, name), i32)))
        p.link_bid = _ptr(keep(g.link_boundary_id, i32))
        for name in ("link_eta", "link_xb", "link_yb", "link_nx", "link_ny"):
            setattr(p, name, _ptr(keep(getattr(g, name), f64)))
        p.lsq_i, p.lsq_j = _ptr(keep(g.lsq_i, i32)), _ptr(keep(g.lsq_j, i32))
        for name in ("lsq_wb", "lsq_wt", "lsq_wx", "lsq_wy"):
            setattr(p, name, _ptr(keep(getattr(g, name), f64)))
        p.lsq_valid = _ptr(keep(g.lsq_valid, i32))
        p.bc_kind, p.bc_mode, p.bc_params = _ptr(keep(kind, i32)), _ptr(keep(mode, i32)), _ptr(keep(params, f64))
        p.traction_x = p.traction_y = None
        self.p = p
        self.f0 = np.zeros((24, g.nx, g.ny))
        self.f1 = np.zeros_like(self.f0)
        self.fpost = np.zeros_like(self.f0)
        self.U = np.zeros((6, g.nx, g.ny))
        self.u = np.zeros((2, g.nx, g.ny))
        self.u_next = np.zeros_like(self.u)
        self.u_star = np.zeros_like(self.u)
        self.P = np.zeros((4, g.nx, g.ny))
        self.sigma = np.zeros_like(self.P)
        self.invalid = np.zeros(1, np.int32)
        self.bc_diag = np.zeros(N)
        self.bc_rhs = np.zeros(2 * N)
        self.time = 0.0
        self.steps = 0

    def _fields(self):
        from curved_lbm import _native

        fl = _native.Fields2D()
        for name in ("f0", "f1", "fpost", "U", "u", "u_next", "u_star", "P", "sigma", "invalid"):
            setattr(fl, name, _ptr(getattr(self, name)))
        fl.clock = None
        return fl

    def initialize_from_numpy(self, *, U, displacement=None, init_order=1,
                              apply_initial_boundaries=True, initial_boundary_time=0.0):
        from curved_lbm.two_d import vector_nonlinear_elastic_warp as v2

        U = np.asarray(U, float)
        disp = np.zeros((2, self.nx, self.ny)) if displacement is None else np.asarray(displacement, float)
        act = self.g.active.astype(bool)
        kw = dict(dx=self.dx, dy=self.dy, dt=self.dt, periodic_x=False, periodic_y=False,
                  source_mode=self.source_mode, source_params=self.source_params)
        if init_order == 1:
            f = v2._equilibrium_np(U, self.material, self.c)
            f -= (0.5 * self.dt / 4.0) * v2._source_np(U, self.source_mode, self.source_params)[None, ...]
        elif init_order == 2:
            f = v2._second_order_populations_np(U, self.material, self.c, **kw)
        else:
            f = v2._second_order_populations_masked_np(U, act, self.material, self.c, **kw)
        f[:, :, ~act] = 0.0
        dm = disp.copy()
        dm[:, ~act] = 0.0
        us = dm - 0.5 * self.dt * U[:2]
        us[:, ~act] = 0.0
        self.f0[...] = f.reshape(24, self.nx, self.ny)
        self.f1[...] = 0.0
        self.fpost[...] = 0.0
        self.u_star[...] = us
        self.time, self.steps = 0.0, 0
        self.refresh()
        if apply_initial_boundaries:
            self.lib.oracle2d_apply_boundary(C.byref(self.p), C.byref(self._fields()),
                                             C.c_double(initial_boundary_time), 1)
            if self.p.kinetic_filter > 0.0:
                self.lib.oracle2d_kinetic_filter(C.byref(self.p), C.byref(self._fields()))
            self.refresh()

    def refresh(self):
        self.lib.oracle2d_refresh(C.byref(self.p), C.byref(self._fields()))

    def step(self):
        fl = self._fields()
        s = _Scratch2(_ptr(self.bc_diag), _ptr(self.bc_rhs))
        self.lib.oracle2d_step(C.byref(self.p), C.byref(fl), C.byref(s), C.c_double(self.time),
                               C.c_int64(self.steps), C.c_int(self.threads))
        self.f0, self.f1 = self.f1, self.f0
        self.time += self.dt
        self.steps += 1

    def run(self, nsteps):
        for _ in range(int(nsteps)):
            self.step()


def build_char_stencil(geometry, tables, link_mask=None) -> dict:
    """Characteristic stencil of the cut links (oracle/char_stencil3d.c), in
    the reference's layout: indices (64, L), weights (4, 64, L), probe_modes
    (L,).  Raises ValueError like the reference for a link without a
    full-rank fit or with inconsistent gradient weights."""
    lib = load()
    g = geometry
    L = int(g.n_links)
    idx = np.full((64, L), -1, np.int32)
    w = np.zeros((4, 64, L))
    modes = np.zeros(L, np.int32)
    status = np.zeros(L, np.int32)
    aid = np.ascontiguousarray(tables["active_id"], dtype=np.int32)
    i32, f64 = np.int32, np.float64
    arr = {k: np.ascontiguousarray(getattr(g, k), dtype=i32) for k in ("link_i", "link_j",
                                                                       "link_k", "link_q")}
    arr.update({k: np.ascontiguousarray(getattr(g, k), dtype=f64) for k in (
        "link_eta", "link_xb", "link_yb", "link_zb", "link_nx", "link_ny", "link_nz")})
    mask = None if link_mask is None else np.ascontiguousarray(link_mask, dtype=np.uint8)
    lib.oracle3d_char_stencil.restype = C.c_int
    bad = lib.oracle3d_char_stencil(
        C.c_int(g.nx), C.c_int(g.ny), C.c_int(g.nz), _ptr(aid), C.c_int(L),
        *(_ptr(arr[k]) for k in ("link_i", "link_j", "link_k", "link_q", "link_eta", "link_xb",
                                 "link_yb", "link_zb", "link_nx", "link_ny", "link_nz")),
        C.c_double(float(g.dx)), _ptr(mask), _ptr(idx), _ptr(w), _ptr(modes), _ptr(status))
    if bad >= 0:
        if status[bad] == 1:
            raise ValueError("local_f needs a full-rank quadratic stencil within three cells; "
                             f"cut links {np.flatnonzero(status == 1)[:8].tolist()}")
        raise ValueError(f"invalid local_f gradient weights near link {bad}")
    return {"indices": idx, "weights": w, "probe_modes": modes}


class Oracle3D:
    """Serial/OpenMP CPU replay of WarpSparseCurvedBoundaryLBM3D (reference C3:3852-4802)."""

    def __init__(self, geometry, *, material, boundary, lattice_speed=5.0, collision_omega=1.8,
                 boundary_reconstruction="bfl", jacobian_floor=1e-12, source_mode="none",
                 source_vector=(0.0,) * 12, damping_gamma=0.0, local_displacement_interval=0,
                 local_displacement_sweeps=1, local_displacement_relax=0.85,
                 local_displacement_boundary_weight=20.0, local_displacement_boundary_id=-1,
                 local_compatibility_interval=0, local_compatibility_blend=0.1,
                 normal_jacobian=None, neumann_solver=None, threads=1, char_stencil=None,
                 **_unused):
        """`char_stencil`: characteristic stencil tables to use (e.g. the ones a
        CUDA solver built), else they are built by oracle/char_stencil3d.c."""
        from curved_lbm import _native
        from curved_lbm.three_d import curved_boundary_warp3d as c3
        from curved_lbm.three_d import geometry3d as g3

        self.lib = load()
        self.g = g = geometry
        self.material = material
        self.threads = int(threads)
        tables = g3._sparse_tables_from_geometry(g)
        self.tables = tables
        n = self.N = int(tables["active_i"].size)
        L = g.n_links
        self.c = float(lattice_speed)
        self.dt = g.dx / self.c
        self.source_mode = c3.source_id(source_mode)
        sp = np.zeros(12)
        if self.source_mode == 1:
            sp[: len(source_vector)] = np.asarray(source_vector, float)[:12]
        elif self.source_mode == 2:
            sp[0] = float(damping_gamma)
        self.source_params = sp
        recon = c3._recon_id(boundary_reconstruction)
        nsolver = c3.neumann_solver_name(neumann_solver, material)
        nj = c3._normal_jacobian_for_material(material, normal_jacobian)
        kind, mode, params = boundary.tables(16)
        ck = boundary.component_kind_table(16)
        clipped = np.clip(g.link_boundary_id, 0, 15).astype(np.int32)
        lck = ck[:, clipped]
        has_neu = bool(L and np.any(lck == 2))
        self._keep = []

        def keep(a, dtype):
            a = np.ascontiguousarray(a, dtype=dtype)
            self._keep.append(a)
            return a

        p = _native.Problem3D()
        p.n_active, p.n_links, p.nx, p.ny, p.nz = n, L, g.nx, g.ny, g.nz
        p.recon, p.normal_solver = recon, 2 if nsolver == "energy" else nj
        p.source_mode = self.source_mode
        char = None
        if recon == 3 and has_neu:
            char = char_stencil if char_stencil is not None else build_char_stencil(
                g, tables, link_mask=np.any(lck == 2, axis=0))
        p.has_char = int(char is not None)
        p.has_tangent_lsq = int(recon == 2)
        p.disp_interval = int(max(0, local_displacement_interval))
        p.disp_sweeps = int(local_displacement_sweeps)
        p.disp_bid = int(local_displacement_boundary_id)
        p.rep_interval = int(max(0, local_compatibility_interval))
        p.dx, p.dy, p.dz, p.dt, p.omega, p.c = g.dx, g.dy, g.dz, self.dt, float(collision_omega), self.c
        for i in range(12):
            p.source[i] = sp[i]
        p.mat = _native.Material(material.id, 0, material.lam, material.mu, material.param0,
                                 material.param1, material.param2, float(jacobian_floor))
        p.relax = float(local_displacement_relax)
        p.weight = float(local_displacement_boundary_weight)
        p.blend = float(local_compatibility_blend)
        i32, f64 = np.int32, np.float64
        p.active_i, p.active_j, p.active_k = (_ptr(keep(tables[k], i32)) for k in ("active_i", "active_j", "active_k"))
        p.neighbor = _ptr(keep(tables["neighbor"], i32))
        p.link_p, p.link_up = _ptr(keep(tables["link_p"], i32)), _ptr(keep(tables["link_upstream"], i32))
        p.link_q, p.link_bid = _ptr(keep(g.link_q, i32)), _ptr(keep(clipped, i32))
        for name in ("link_eta", "link_xb", "link_yb", "link_zb", "link_nx", "link_ny", "link_nz"):
            setattr(p, name, _ptr(keep(getattr(g, name), f64)))
        if recon == 2:
            lsq = g3._build_sparse_tangent_lsq_weights(g, tables)
            p.lsq_p, p.lsq_wt1 = _ptr(keep(lsq["lsq_p"], i32)), _ptr(keep(lsq["lsq_wt1"], f64))
            p.lsq_wt2, p.lsq_valid = _ptr(keep(lsq["lsq_wt2"], f64)), _ptr(keep(lsq["lsq_valid"], i32))
        if char is not None:
            p.char_idx, p.char_w = _ptr(keep(char["indices"], i32)), _ptr(keep(char["weights"], f64))
        p.bc_kind, p.bc_mode = _ptr(keep(kind, i32)), _ptr(keep(mode, i32))
        p.bc_comp_kind, p.bc_params = _ptr(keep(ck, i32)), _ptr(keep(params, f64))
        p.dyn_enabled = p.dyn_traction = None
        self.p = p
        self.f0 = np.zeros((72, n))
        self.f1 = np.zeros_like(self.f0)
        self.U = np.zeros((12, n))
        self.u = np.zeros((3, n))
        self.u_next = np.zeros_like(self.u)
        self.u_star = np.zeros_like(self.u)
        self.link_kind = np.zeros(L, np.int32)
        self.link_comp_kind = np.zeros((3, L), np.int32)
        self.link_bv = np.zeros((3, L))
        self.link_Fb = np.zeros((9, L))
        self.link_Pb = np.zeros((9, L))
        self.char_state = np.zeros((4, 12, L)) if char is not None else None
        self.invalid = np.zeros(1, np.int32)
        self.bc_diag = np.zeros(3 * n)
        self.bc_rhs = np.zeros(3 * n)
        self.time, self.steps = 0.0, 0

    def _fields(self):
        from curved_lbm import _native

        fl = _native.Fields3D()
        for name in ("f0", "f1", "U", "u", "u_next", "u_star", "link_kind", "link_comp_kind",
                     "link_bv", "link_Fb", "link_Pb", "char_state", "invalid"):
            setattr(fl, name, _ptr(getattr(self, name)))
        fl.clock = None
        return fl

    def initialize_identity(self):
        from curved_lbm.three_d import vector_nonlinear_elastic_warp3d as v3

        n = self.N
        U = np.zeros((12, n))
        U[3] = U[7] = U[11] = 1.0
        f = v3._equilibrium_np(U, self.material, self.c)
        src = v3._source_np(U, self.source_mode, self.source_params)
        f -= 0.5 * self.dt / 6.0 * src[None, ...]
        self.f0[...] = f.reshape(72, n)
        self.f1[...] = 0.0
        self.u_star[...] = -0.5 * self.dt * U[:3]
        self.time, self.steps = 0.0, 0
        self.refresh()
        self.lib.oracle3d_apply_boundary(C.byref(self.p), C.byref(self._fields()), C.c_double(0.0), 1)
        self.refresh()
        self.u_star[...] = np.zeros((3, n)) - 0.5 * self.dt * self.U[:3]
        self.refresh()

    def refresh(self):
        self.lib.oracle3d_refresh(C.byref(self.p), C.byref(self._fields()))

    def step(self):
        fl = self._fields()
        s = _Scratch2(_ptr(self.bc_diag), _ptr(self.bc_rhs))
        self.lib.oracle3d_step(C.byref(self.p), C.byref(fl), C.byref(s), C.c_double(self.time),
                               C.c_int64(self.steps), C.c_int(self.threads))
        self.f0, self.f1 = self.f1, self.f0
        self.time += self.dt
        self.steps += 1

    def run(self, nsteps):
        for _ in range(int(nsteps)):
            self.step()


def set_signatures():
    lib = load()
    for name in ("oracle2d_step", "oracle2d_apply_boundary", "oracle2d_refresh", "oracle3d_step",
                 "oracle3d_apply_boundary", "oracle3d_refresh"):
        getattr(lib, name).restype = C.c_int
    return lib
