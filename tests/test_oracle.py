"""Pin the CPU oracle to the reference: it must reproduce every fixture the
reference produced (tests/golden), at the same tolerance the GPU path meets.

Runs on CPU only (no GPU needed).
"""

from __future__ import annotations

import numpy as np
import pytest

import cases

RTOL = 1e-12
ATOL = 1e-15
GOLD2 = ["g2_affine_compat", "g2_traction_localf", "g2_bfl_mixed_fd", "g2_energy_intervals"]
GOLD3 = ["g3_shell_localf", "g3_shell_bfl_fd", "g3_shell_compat"]
# one case per material law other than neo-Hooke (tests/golden/make_golden.py)
GOLD2 += [f"g2_mat_{m}" for m in ("svk", "log_neo_hooke", "mooney_rivlin", "yeoh", "gent",
                                   "sugiyama_svk")]
GOLD2 += ["g2_mrt_ghost", "g2_kinetic_filter", "g2_mrt_filter"]
GOLD2 += ["g2_lsq_bfl", "g2_compat_bfl_traction", "g2_local_char2", "g2_local_f_bfl"]
GOLD3 += ["g3_mixed_localf", "g3_mixed_fd", "g3_mixed_energy"]
GOLD3 += ["g3_shell_halfway", "g3_shell_localf_bfl"]
GOLD3 += [f"g3_mat_{m}" for m in ("svk", "log_neo_hooke", "mooney_rivlin", "yeoh", "gent",
                                   "sph_neo_hooke")]


def close(name, got, ref, rtol=RTOL, atol=ATOL):
    got, ref = np.asarray(got), np.asarray(ref)
    assert got.shape == ref.shape, (name, got.shape, ref.shape)
    err = np.abs(got - ref)
    bad = err > atol + rtol * np.abs(ref)
    assert not bad.any(), f"{name}: {int(bad.sum())} off, max err {float(err.max()):.3e}"


def oracle_2d(cfg, **kw):
    from curved_lbm.two_d import curved_boundary_warp as c2
    from curved_lbm.two_d.vector_nonlinear_elastic_warp import WarpHyperelasticMaterial
    from oracle.oracle import Oracle2D

    g = cases.geometry_2d(cfg["geometry"])
    m = cfg["material"]
    mat = WarpHyperelasticMaterial.from_poisson(m["model"], m["poisson"], mu=m["mu"], **m.get("extra", {}))
    spec = c2.CurvedBoundarySpec(**cases.boundary_kwargs(cfg["boundary"]))
    return Oracle2D(g, material=mat, boundary=spec, **cfg["solver"], **kw)


def oracle_3d(cfg, **kw):
    from curved_lbm.three_d import curved_boundary_warp3d as c3
    from oracle.oracle import Oracle3D

    g = cases.geometry_3d(cfg["geometry"])
    m = cfg["material"]
    mat = c3.WarpHyperelasticMaterial3D.from_poisson(m["model"], m["poisson"], mu=m["mu"], **m.get("extra", {}))
    spec = c3.CurvedBoundarySpec3D(**cases.boundary_kwargs(cfg["boundary"]))
    return Oracle3D(g, material=mat, boundary=spec, **cfg["solver"], **kw)


@pytest.mark.parametrize("name", GOLD2)
@pytest.mark.parametrize("threads", [1, 4])
def test_oracle_2d_reproduces_reference(golden_dir, name, threads):
    d, cfg = cases.load(golden_dir / f"{name}.npz")
    o = oracle_2d(cfg, threads=threads)
    U0, disp0 = cases.initial_state_2d(cfg["init"], o.g)
    o.initialize_from_numpy(U=U0, displacement=disp0, init_order=cfg["init"]["init_order"])
    close("f0_init", o.f0, d["f0_init"])
    close("ustar_init", o.u_star, d["ustar_init"])
    o.run(cfg["steps"])
    close("f0", o.f0, d["f0"])
    close("u_star", o.u_star, d["ustar"])
    close("U_step", o.U, d["U_step"])
    close("u_step", o.u, d["u_step"])
    o.refresh()
    close("U", o.U, d["U"])
    close("u", o.u, d["u"])
    close("P", o.P, d["P"])
    close("sigma", o.sigma, d["sigma"])


@pytest.mark.parametrize("name", GOLD3)
def test_oracle_3d_reproduces_reference(golden_dir, name):
    """The time step on the reference's own characteristic stencil tables
    (stored in the fixture; the builders are pinned in test_char_stencil.py)."""
    d, cfg = cases.load(golden_dir / f"{name}.npz")
    kw = {}
    if "char_indices" in d.files:
        kw["char_stencil"] = {"indices": d["char_indices"], "weights": d["char_weights"],
                              "probe_modes": d["char_modes"]}
    o = oracle_3d(cfg, threads=2, **kw)
    o.initialize_identity()
    close("f0_init", o.f0, d["f0_init"])
    close("ustar_init", o.u_star, d["ustar_init"])
    o.run(cfg["steps"])
    close("f0", o.f0, d["f0"])
    close("u_star", o.u_star, d["ustar"])
    close("link_Fb", o.link_Fb, d["link_Fb"])
    close("link_Pb", o.link_Pb, d["link_Pb"])
    close("link_bv", o.link_bv, d["link_bv"])
    if o.char_state is not None:
        close("char_state", o.char_state, d["char_state"])
    o.refresh()
    close("U", o.U, d["U"])
    close("u", o.u, d["u"])


def test_oracle_warp_regression_fixture(golden_dir):
    """The reference's Warp-produced 3-D BFL regression (25 steps, atol 1e-13)."""
    from curved_lbm.three_d import curved_boundary_warp3d as cb
    from oracle.oracle import Oracle3D

    ref = np.load(golden_dir / "dirichlet_bfl_3d_reference.npz")
    g = cb.CurvedBoundaryGeometry3D.sphere(nx=20, ny=20, nz=20, radius=0.35)
    mat = cb.WarpHyperelasticMaterial3D.from_poisson("neo_hooke", 0.2, mu=1.0)
    spec = cb.CurvedBoundarySpec3D(kind="neumann", component_kinds=("dirichlet",) * 3,
                                   value_mode=1, params=(0.001, 0.002, -0.001))
    o = Oracle3D(g, material=mat, boundary=spec, boundary_reconstruction="local_f",
                 lattice_speed=10.0, collision_omega=1.8)
    from curved_lbm.three_d import vector_nonlinear_elastic_warp3d as v3

    U = ref["U"]
    f = v3._equilibrium_np(U, mat, 10.0)
    o.f0[...] = f.reshape(72, -1)
    o.u_star[...] = -0.5 * o.dt * U[:3]
    o.refresh()
    o.run(25)
    np.testing.assert_allclose(o.f0, ref["f25"], rtol=0, atol=1e-13)
