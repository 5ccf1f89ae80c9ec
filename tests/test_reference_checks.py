"""The reference's own behavioural tests, restated for this package.

tests/test_gradients.py (rest state under local_f traction closure) and
tests/test_initial_boundary_buffers.py (in-place boundary pass equals the
frozen-source evaluation) of the reference, plus its characteristic
population formula check (tests/test_characteristics.py:120-232) for the
all-Neumann component case.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_zero_traction_rest_state_is_preserved():
    from curved_lbm.two_d import curved_boundary_warp as c2

    n = 24
    g = c2.CurvedBoundaryGeometry.circle(nx=n, ny=n, radius=0.35)
    m = c2.WarpHyperelasticMaterial.from_poisson("neo_hooke", 0.2, mu=1.0)
    s = c2.WarpCurvedBoundaryLBM2D(
        g, material=m, boundary=c2.CurvedBoundarySpec(kind="neumann"),
        boundary_reconstruction="local_f", lattice_speed=10.0, collision_omega=1.8,
        local_displacement_interval=1, local_compatibility_interval=1,
        local_compatibility_blend=0.5)
    U = np.zeros((6, n, n))
    U[2] = U[5] = 1.0
    s.initialize_from_numpy(U=U, displacement=np.zeros((2, n, n)), apply_initial_boundaries=False)
    for _ in range(5):
        s.step()
    s.refresh_current()
    act = s.active_np.astype(bool)
    assert float(np.max(np.abs(s.system_state()[:, act] - U[:, act]))) < 1e-11


@pytest.mark.parametrize("storage", ["2d", "3d_sparse"])
def test_in_place_boundary_matches_frozen_source(storage):
    import torch

    if storage == "2d":
        from curved_lbm.two_d import curved_boundary_warp as c2

        geometry = c2.CurvedBoundaryGeometry.circle(nx=8, ny=8, radius=0.12)
        material = c2.WarpHyperelasticMaterial.from_poisson("neo_hooke", 0.2, mu=1)
        boundary = c2.CurvedBoundarySpec(kind="dirichlet", value_mode=c2.VALUE_CONSTANT,
                                         params=(0.001, -0.002))
        solver = c2.WarpCurvedBoundaryLBM2D(geometry, material=material, boundary=boundary,
                                            boundary_reconstruction="bfl", lattice_speed=10,
                                            collision_omega=1.8)
    else:
        from curved_lbm.three_d import curved_boundary_warp3d as c3

        geometry = c3.CurvedBoundaryGeometry3D.sphere(nx=8, ny=8, nz=8, radius=0.12)
        material = c3.WarpHyperelasticMaterial3D.from_poisson("neo_hooke", 0.2, mu=1)
        boundary = c3.CurvedBoundarySpec3D(kind="dirichlet",
                                           value_mode=c3.CURVED3D_VALUE_CONSTANT_VECTOR,
                                           params=(0.001, -0.002, 0.003))
        solver = c3.WarpSparseCurvedBoundaryLBM3D(geometry, material=material, boundary=boundary,
                                                  boundary_reconstruction="bfl", lattice_speed=10,
                                                  collision_omega=1.8)
    before = solver.f0.cpu().numpy() + np.random.default_rng(501).normal(0, 0.001, solver.f0.shape)
    frozen = torch.as_tensor(before, device=solver.f0.device)
    solver.f0.copy_(frozen)
    if hasattr(solver, "fpost"):
        solver.fpost.copy_(frozen)
    solver.f1.fill_(float("nan"))
    solver.apply_boundary_reconstruction(0.03, in_place=False)
    separate = solver.f1.cpu().numpy()
    written = np.isfinite(separate)
    assert written.any()
    expected = before.copy()
    expected[written] = separate[written]
    solver.f0.copy_(frozen)
    solver.apply_boundary_reconstruction(0.03, in_place=True)
    np.testing.assert_array_equal(solver.f0.cpu().numpy(), expected)


def _flux(U, material, axis, cb):
    P = cb._first_piola_np(U[3:].reshape(3, 3), material)
    out = np.zeros(12)
    out[:3] = -P[:, axis]
    out[3:].reshape(3, 3)[:, axis] = -U[:3]
    return out


def _derivative(U, W, material, axis, cb):
    eps = 2e-6 / max(1.0, np.max(np.abs(W)))
    return (_flux(U + eps * W, material, axis, cb) - _flux(U - eps * W, material, axis, cb)) / (2 * eps)


def test_characteristic_population_formula(golden_dir):
    """Newton traction and incoming characteristic populations, all-Neumann rows."""
    import torch

    from curved_lbm.three_d import curved_boundary_warp3d as cb

    g = cb.CurvedBoundaryGeometry3D.sphere(nx=20, ny=20, nz=20, radius=0.35)
    original = np.load(golden_dir / "dirichlet_bfl_3d_reference.npz")
    material = cb.WarpHyperelasticMaterial3D.from_poisson("neo_hooke", 0.2, mu=1.0)
    boundary = cb.CurvedBoundarySpec3D(kind="neumann", component_kinds=("neumann",) * 3,
                                       value_mode=cb.CURVED3D_VALUE_CONSTANT_VECTOR,
                                       params=(0.001, 0.002, -0.001))
    s = cb.WarpCurvedBoundaryLBM3D(g, material=material, boundary=boundary,
                                   boundary_reconstruction="local_f", lattice_speed=10.0,
                                   source_mode="damping", damping_gamma=0.7)
    x, y, z = s.active_coordinates()
    U = np.zeros((12, s.n_active))
    U[0], U[1], U[2] = 0.03 * x * y, 0.02 * y * z, -0.01 * z * x
    U[3], U[7], U[11] = 1 + 0.01 * x, 1 + 0.01 * y, 1 + 0.01 * z
    U[4] = 0.003 * y
    s.initialize_from_numpy(U=U, displacement=np.zeros((3, s.n_active)),
                            apply_initial_boundaries=False)
    s.f0.copy_(torch.as_tensor(original["f_source"], device=s.f0.device))
    s.apply_boundary_reconstruction(0.03)
    state = s.char_state.cpu().numpy()
    Fb, Pb, bv = s.link_Fb.cpu().numpy(), s.link_Pb.cpu().numpy(), s.link_bv.cpu().numpy()
    current, output, nodes = s.U.cpu().numpy(), s.f1.cpu().numpy(), s.link_p.cpu().numpy()
    normal = np.array((g.link_nx, g.link_ny, g.link_nz))
    traction = np.einsum("ijl,jl->il", Pb.reshape(3, 3, -1), normal)
    np.testing.assert_allclose(traction, bv, atol=2e-9, rtol=1e-7)
    for ell in np.linspace(0, g.n_links - 1, 31, dtype=int):
        qi = (g.link_q[ell] + 3) % 6
        d = cb.DIRS3[qi].astype(float)
        Ub = np.r_[current[:3, nodes[ell]], Fb[:, ell]]
        G = state[1:, :, ell]
        Uc = Ub + g.link_eta[ell] * s.dt * s.lattice_speed * (d @ G)
        B = np.zeros(12)
        B[:3] = -0.7 * Uc[:3]
        w = B - sum(_derivative(Uc, G[a], material, a, cb) for a in range(3)) + s.lattice_speed * (d @ G)
        feq = (Uc + 3 / s.lattice_speed * sum(d[a] * _flux(Uc, material, a, cb) for a in range(3))) / 6
        deq = (w + 3 / s.lattice_speed * sum(d[a] * _derivative(Uc, w, material, a, cb) for a in range(3))) / 6
        expected = feq - s.dt / s.collision_omega * deq + s.dt * (1 / s.collision_omega - 0.5) * B / 6
        np.testing.assert_allclose(output[12 * qi: 12 * (qi + 1), nodes[ell]], expected,
                                   rtol=2e-8, atol=2e-10)
    before = s.f1.cpu().numpy().copy()
    s.f0.fill_(123.0)
    s.apply_boundary_reconstruction(0.03)
    after = s.f1.cpu().numpy()
    slots = 12 * ((g.link_q + 3) % 6)[:, None] + np.arange(12)[None, :]
    np.testing.assert_array_equal(before[slots, nodes[:, None]], after[slots, nodes[:, None]])
