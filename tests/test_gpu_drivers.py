"""Device drivers against the reference's converged solutions.

C1 (subsonic channel 40x10x10, M_inf 0.5): the reference ``solve_subsonic``
converged potential (golden fixture, pyamg swapped for spilu there); the
north-star bar is converged Cp within 1e-8.
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
