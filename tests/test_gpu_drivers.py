"""Device drivers against the reference's converged solutions.

C1 (subsonic channel 40x10x10, M_inf 0.5): the reference ``solve_subsonic``
converged potential (golden fixture, pyamg swapped for spilu there); the
parity bar is converged Cp within 1e-8.
"""

import numpy as np
import pytest

from conftest import has_cuda

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]


def test_subsonic_picard_matches_reference(picard_golden):
    import torch
    from up3d_b200.kernels.jacobian import PicardOperator
    from up3d_b200.physics.isentropic import pressure_coefficient_field
    from up3d_b200.solve.picard import solve_subsonic
    g = picard_golden
    nodes, elements, dn = g["nodes"], g["elements"], g["dirichlet_nodes"]
    res = solve_subsonic(nodes, elements, dn, nodes[dn, 0], float(g["m_inf"]))
    assert res["converged"]
    assert res["residual_history"][-1] < 1e-10
    op = PicardOperator(torch.from_numpy(nodes), torch.from_numpy(elements))
    _, q2 = op.velocities(torch.from_numpy(res["phi"]).cuda())
    cp = pressure_coefficient_field(q2, float(g["m_inf"])).cpu().numpy()
    err = np.abs(cp - g["cp"]).max()
    assert err < 1e-8, f"converged Cp error {err:.2e}"
    assert np.abs(res["phi"] - g["phi"]).max() < 1e-8


def test_transonic_newton_converges_on_reference_equations():
    """Mach continuation 0.70 -> 0.85 on a 40x12x10 bump channel (bump 0.08):
    the device Newton (exact Jacobian, GMRES + AMG, line search, frozen
    finish) reaches |R_free| < 1e-10 with a supersonic pocket.  The converged
    potential satisfies the reference's discrete equations as the solver
    finished them: with the frozen (upstream, branch) state when the finish
    froze (pyfp3d/solve/newton.py accepts a frozen convergence whose live
    residual stops improving), else the live ones.  The live residual the
    solver reports equals the oracle's at the same potential."""
    import torch
    from oracle import oracle as O
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.solve.newton import ChannelWorkspace, solve_newton_transonic
    mesh = bump_channel(40, 12, 10, amplitude=0.08, seed=0)
    ws = ChannelWorkspace(mesh.nodes, mesh.elements, mesh.dirichlet_nodes)
    res = solve_newton_transonic(ws, 0.85, m_start=0.70, dm=0.05)
    assert res["converged"], res["level_history"]
    assert res["residual_history"][-1] < 1e-10
    assert res["n_supersonic"] > 0
    phi = res["phi"].cpu().numpy()
    op = O.PicardOperator(mesh.nodes, mesh.elements)
    upw = O.UpwindOperator(mesh.nodes, mesh.elements)
    free = np.setdiff1d(np.arange(mesh.n_nodes), mesh.dirichlet_nodes)
    live = O.chain(op, upw, phi, 0.85, jacobian=False)
    r_live = np.abs(live["R"][free]).max()
    if res["froze"]:
        up, br = (x.cpu().numpy() for x in res["frozen_state"])
        rt = upw.rho_tilde_frozen(live["q2l"], live["rho"], up, br, 0.85, O.UPWIND_C, O.M_CRIT)
        R = op.assemble_residual(phi, rt)
        assert np.abs(R[free]).max() < 2e-10
        if res["residual_unfrozen"] is not None:
            assert abs(r_live - res["residual_unfrozen"]) <= 1e-9 * max(r_live, 1e-300) + 1e-18
    else:
        assert r_live < 2e-10
        assert live["n_supersonic"] == res["n_supersonic"]


def test_mixed_precision_newton_matches_fp64():
    """Newton with FP32 Jacobian SpMV and FP32 AMG inside FP64-refined
    GMRES reaches the FP64 solve's potential (residual, update and test in
    FP64) on a 40x12x10 channel at M0.80."""
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.solve.newton import ChannelWorkspace, solve_newton_transonic
    mesh = bump_channel(40, 12, 10, amplitude=0.08, seed=0)
    ws = ChannelWorkspace(mesh.nodes, mesh.elements, mesh.dirichlet_nodes)
    r64 = solve_newton_transonic(ws, 0.80, m_start=0.70, dm=0.05)
    ws2 = ChannelWorkspace(mesh.nodes, mesh.elements, mesh.dirichlet_nodes)
    r32 = solve_newton_transonic(ws2, 0.80, m_start=0.70, dm=0.05, precision="mixed")
    assert r64["converged"] and r32["converged"]
    assert r32["residual_history"][-1] < 1e-10 and r32["n_refinements"] > 0
    assert np.abs(r32["phi"].cpu().numpy() - r64["phi"].cpu().numpy()).max() < 1e-8
