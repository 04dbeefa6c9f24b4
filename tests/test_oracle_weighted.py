"""The oracle's weighted upwind modes (face normals, BFS neighbourhoods,
the streamline-kernel and face-blend rho~) against the reference's outputs
on the same meshes and states (tests/golden/weighted_upwind.npz, made by
tests/golden/make_golden.py)."""

import numpy as np
import pytest

from conftest import GOLDEN, REL_TOL, rel_err

M_CRIT, UPWIND_C, RHO_FLOOR, M_CAP, GAMMA = 0.95, 1.5, 0.05, 3.0, 1.4
PARAMS = {
    "default": dict(p_weight=3.0, reach_frac=1.0, reach_gain_max=4.0, nbr_depth=3,
                    sigma_s_frac=0.35, sigma_p_frac=0.35),
    "alt": dict(p_weight=2.0, reach_frac=0.8, reach_gain_max=3.0, nbr_depth=2,
                sigma_s_frac=0.5, sigma_p_frac=0.25),
}


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "weighted_upwind.npz")


def states(gold):
    return sorted({k.split("/")[1] for k in gold.files if k.startswith("state/")})


def test_face_normals(gold):
    from oracle import oracle as O
    fn = O.face_normals(gold["mesh/nodes"], gold["mesh/elements"])
    ref = gold["mesh/face_normals"]
    assert np.abs(fn - ref).max() < 1e-14
    assert np.allclose(np.linalg.norm(fn, axis=2), 1.0, atol=1e-12)


@pytest.mark.parametrize("pname", ["default", "alt"])
def test_neighborhoods_exact(gold, pname):
    from oracle import oracle as O
    fnb = O.face_adjacency(gold["mesh/elements"])
    off, idx = O.build_upstream_neighborhoods(fnb, PARAMS[pname]["nbr_depth"])
    assert np.array_equal(off, gold[f"{pname}/nb_off"])
    assert np.array_equal(idx, gold[f"{pname}/nb_idx"])


@pytest.mark.parametrize("pname", ["default", "alt"])
@pytest.mark.parametrize("mode", ["kernel", "blend"])
def test_weighted_rho_tilde(gold, pname, mode):
    from oracle import oracle as O
    nodes, elements = gold["mesh/nodes"], gold["mesh/elements"]
    op = O.PicardOperator(nodes, elements)
    upw = O.UpwindOperator(nodes, elements, weighted=True, mode=mode, **PARAMS[pname])
    for label in states(gold):
        phi, m_inf = gold[f"state/{label}/phi"], float(gold[f"state/{label}/m_inf"])
        grad, q2 = op.velocities(phi)
        q2l = O.limit_q2_field(q2, m_inf, M_CAP, GAMMA)
        rho = O.density_field(q2l, m_inf, GAMMA)
        rt = upw.rho_tilde(grad, q2l, rho, m_inf, UPWIND_C, M_CRIT, GAMMA, RHO_FLOOR)
        key = f"{pname}/{mode}/{label}"
        assert rel_err(rt, gold[f"{key}/rho_tilde"]) < REL_TOL, key
        assert rel_err(upw.nu, gold[f"{key}/nu"]) < REL_TOL, key
        assert upw.n_supersonic == int(gold[f"{key}/n_supersonic"]), key
        assert upw.n_floored == int(gold[f"{key}/n_floored"]), key
        assert abs(upw.nu_max - float(gold[f"{key}/nu_max"])) <= 1e-12 * max(1.0, upw.nu_max)
