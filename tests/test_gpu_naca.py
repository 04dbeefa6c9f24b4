"""Device lifting Newton on the reference's NACA0012 2.5D coarse mesh, cut
by the reference's own cut_wake (tests/golden/naca_coarse.npz): the
converged potential, circulation, wall Cp and lift against the reference's
solve_newton_lifting and wall_force_coefficients (solve/newton.py:516-1141,
post/surface.py:309-363) -- converged Cp within 1e-8."""

import numpy as np
import pytest

from conftest import GOLDEN
from test_mesh_reader import _mesh, naca_cut

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def naca():
    return np.load(GOLDEN / "naca_coarse.npz")


@pytest.mark.parametrize("case", ["m05", "m07"])
def test_gpu_naca_lifting_matches_reference(naca, case):
    from up3d_b200.post.surface import wall_force_coefficients
    from up3d_b200.solve.lifting import solve_newton_lifting
    if case == "m07":
        # the whole chain on this side: the mesh arrays as read from the
        # .msh, cut by this library's cut_wake (equal to the reference's)
        from up3d_b200.mesh.wake_cut import cut_wake
        mc, wc = cut_wake(_mesh(naca))
    else:
        mc, wc = naca_cut(naca)
    m_inf, alpha = float(naca[case + "/m_inf"]), float(naca[case + "/alpha_deg"])
    res = solve_newton_lifting(mc, wc, m_inf, alpha_deg=alpha, n_picard_seed=0)
    assert res["converged"]
    phi = res["phi"].cpu().numpy()
    assert np.max(np.abs(phi - naca[case + "/phi"])) <= 1e-9
    assert np.max(np.abs(res["gamma"].cpu().numpy() - naca[case + "/gamma"])) <= 1e-9
    assert res["n_nu_active"] == int(naca[case + "/n_nu_active"])
    f = wall_force_coefficients(mc.nodes, mc.elements, np.asarray(mc.boundary_faces["wall"]), res["phi"],
                                alpha_deg=alpha, m_inf=m_inf)
    cp = f["cp_tri"].cpu().numpy() if hasattr(f["cp_tri"], "cpu") else np.asarray(f["cp_tri"])
    assert np.max(np.abs(cp - naca[case + "/cp_tri"])) <= 1e-8
    assert abs(float(f["cl"]) - float(naca[case + "/cl"])) <= 1e-10


@pytest.mark.parametrize("tag", ["plain", "taper"])
def test_gpu_naca_pressure_kutta_matches_reference(naca, tag):
    """kutta_estimator="pressure" (constraints/te_pressure.py, the
    eliminated step of solve/newton.py:459-502), untapered and with the
    tip-taper blend: the reference's converged solution and frozen
    scaling (tests/golden/te_pressure.npz)."""
    from up3d_b200.solve.lifting import solve_newton_lifting
    g = np.load(GOLDEN / "te_pressure.npz")
    mc, wc = naca_cut(naca)
    taper = None if tag == "plain" else np.array([0.7])
    res = solve_newton_lifting(mc, wc, 0.5, alpha_deg=1.25, n_picard_seed=0, kutta_estimator="pressure",
                               tip_taper=taper)
    assert res["converged"]
    assert np.max(np.abs(res["kutta_sigma"] - g[tag + "/kutta_sigma"])) <= 1e-12 * np.max(g[tag + "/kutta_sigma"])
    assert np.max(np.abs(res["phi"].cpu().numpy() - g[tag + "/phi"])) <= 1e-9
    assert np.max(np.abs(res["gamma"].cpu().numpy() - g[tag + "/gamma"])) <= 1e-9


def test_gpu_naca_transonic_recipe_matches_reference(naca):
    """The reference's own transonic case (M0.80, alpha 1.25 deg, Mach ramp
    from 0.70 with its committed recipe: dm 0.025, freeze 1e-6, direct
    steps; cases/analysis/a1_solver_bottleneck, published 5 levels, 57
    Newton steps, Gamma 0.233826): the same level sequence and the
    reference's converged solution."""
    from up3d_b200.solve.lifting import solve_newton_transonic
    mc, wc = naca_cut(naca)
    res = solve_newton_transonic(mc, wc, 0.8, 1.25, m_start=0.70, dm=0.025, dm_min=0.003, freeze_tol=1e-6,
                                 newton_kw=dict(freeze_refresh_max=8, precond="direct", n_newton_max=60,
                                                n_picard_seed=0))
    assert res["converged"]
    ref = naca["m08/levels"]
    got = np.array([[m, n, r] for m, n, r in res["level_history"]])
    assert np.allclose(got[:, 0], ref[:, 0])
    assert np.all(np.abs(got[:, 1] - ref[:, 1]) <= 2)
    assert abs(float(res["gamma"][0]) - float(naca["m08/gamma"][0])) <= 1e-8
    assert np.max(np.abs(res["phi"].cpu().numpy() - naca["m08/phi"])) <= 1e-8
