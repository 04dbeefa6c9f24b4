"""The pressure-equality Kutta estimator's control volumes
(pyfp3d/constraints/te_pressure.py, TEControlVolumes) on the NACA0012
coarse cut against the reference's own (tests/golden/te_pressure.npz),
with the element geometry from the oracle (the device's B is the same
bits: the geometry parity tests)."""

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN


@pytest.fixture(scope="module")
def cvs():
    from oracle import oracle as O
    from up3d_b200.constraints.dirichlet import FarfieldBasis
    from up3d_b200.constraints.te_pressure import TEControlVolumes
    from up3d_b200.mesh.wake_cut import load_cut
    mc, wc = load_cut(np.load(GOLDEN / "naca_coarse.npz"))
    B, V = O.element_geometry(mc.nodes, mc.elements)
    basis = FarfieldBasis(mc, wc, 1.25)
    return TEControlVolumes(mc, wc, dirichlet_nodes=basis.dir_cut, geometry=(B, V))


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "te_pressure.npz")


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_te_control_volumes_match_reference(cvs, gold):
    phi = gold["phi"]
    qu, ql = cvs.te_velocities(phi)
    # B from the oracle restatement of precompute_element_geometry: equal to
    # the reference's to a few ulps
    assert _rel(qu, gold["qu"]) <= 1e-13 and _rel(ql, gold["ql"]) <= 1e-13
    # F_raw is a difference of two O(1) squares: compare on their scale
    scale = float(np.max(np.sum(gold["qu"] ** 2, axis=1)))
    assert np.max(np.abs(cvs.residual_stations(phi) - gold["F_raw"])) <= 1e-13 * scale
    Kp, D = cvs.newton_rows(phi)
    K_ref = sp.csr_matrix((gold["Kp_data"], gold["Kp_indices"], gold["Kp_indptr"]), shape=Kp.shape)
    assert _rel(Kp.toarray(), K_ref.toarray()) <= 1e-13
    assert _rel(D, gold["D"]) <= 1e-13
    assert _rel(cvs.gamma_jacobian(phi, mode="frozen"), gold["D_frozen"]) <= 1e-13
    gamma = np.load(GOLDEN / "naca_coarse.npz")["m05/gamma"] * 0.9
    assert np.max(np.abs(cvs.implied_targets(phi, gamma) - gold["implied"])) <= 1e-12
    st = cvs.fan_stats()
    assert st["n_te"] == 2 and st["fan_u_min"] >= 1 and st["fan_l_min"] >= 1


def test_te_control_volumes_refuse_far_field_dofs(cvs):
    from oracle import oracle as O
    from up3d_b200.constraints.te_pressure import TEControlVolumes
    from up3d_b200.mesh.wake_cut import load_cut
    mc, wc = load_cut(np.load(GOLDEN / "naca_coarse.npz"))
    B, V = O.element_geometry(mc.nodes, mc.elements)
    with pytest.raises(AssertionError):
        TEControlVolumes(mc, wc, dirichlet_nodes=cvs.dofs[:1], geometry=(B, V))
    with pytest.raises(ValueError):
        TEControlVolumes(mc, wc, wall_tag="nope", geometry=(B, V))
