"""The coupled (phi, Gamma) lifting Newton system against the reference's
own NewtonWorkspace / solve_newton_lifting (tests/golden/lifting_newton.npz,
solve/newton.py:97-1141, probe Kutta estimator): the synthetic lifting cut
of the channel, the host far-field split, basis and Kutta row, and the
oracle's eval_residual, coupled blocks and exact-step Newton solve."""

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN

CASES = ["sub", "trans"]


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "lifting_newton.npz")


def _case(gold, name):
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.mesh.wake_cut import cut_channel_sheet
    g = {k.split("/", 1)[1]: gold[k] for k in gold.files if k.startswith(name + "/")}
    cut = cut_channel_sheet(bump_channel(*tuple(int(v) for v in g["shape"]), amplitude=0.08, seed=3),
                            normal="y")
    return g, cut


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", CASES)
def test_lifting_cut_and_farfield_basis_match_reference(gold, name):
    from up3d_b200.constraints.dirichlet import FarfieldBasis, kutta_row
    from up3d_b200.mesh.wake_cut import channel_vortex_center
    g, cut = _case(gold, name)
    assert np.array_equal(cut.nodes, g["nodes"])
    assert np.array_equal(cut.elements, g["elements"])
    assert np.array_equal(cut.boundary_faces["farfield"], g["farfield_faces"])
    vc = channel_vortex_center(cut)
    assert np.array_equal(np.array(vc), g["vortex_center"])
    basis = FarfieldBasis(cut, cut.wc, float(g["alpha_deg"]), 1.0, vc, bool(g["spanwise"]))
    assert np.array_equal(basis.dir_red, g["dir_red"])
    assert np.array_equal(basis.free, g["free"])
    vals0, V = basis.at_mach(float(np.sqrt(1.0 - float(g["m_inf"]) ** 2)))
    assert np.array_equal(vals0, g["vals0_red"])
    assert np.array_equal(V, g["V_red"])
    K = kutta_row(cut.wc, basis.is_dir)
    K_ref = sp.csr_matrix((g["K_data"], g["K_indices"], g["K_indptr"]), shape=(cut.wc.n_stations, len(basis.free)))
    assert np.array_equal(K[:, basis.free].toarray(), K_ref.toarray())
    assert K[:, basis.dir_red].nnz == 0


def test_kutta_row_rejects_far_field_probe(gold):
    from up3d_b200.constraints.dirichlet import kutta_row
    g, cut = _case(gold, "sub")
    is_dir = np.zeros(cut.wc.n_nodes_orig, dtype=bool)
    is_dir[cut.wc.kutta_upper[0]] = True
    with pytest.raises(ValueError):
        kutta_row(cut.wc, is_dir)


def _system(g, cut):
    from oracle import oracle as O
    return O.LiftingSystem(g["nodes"], g["elements"], cut.wc, g["dir_red"], g["vals0_red"], g["V_red"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_lifting_residual_and_blocks_match_reference(gold, name):
    g, cut = _case(gold, name)
    sysm = _system(g, cut)
    m_inf = float(g["m_inf"])
    R, F, st = sysm.eval_residual(g["seed_phi_free"], g["seed_gamma"], m_inf)
    assert np.array_equal(st["phi_cut"], g["seed_phi_cut"])
    assert _rel(R, g["seed_R_free"]) <= 1e-12
    assert _rel(F, g["seed_F"]) <= 1e-12
    assert st["n_supersonic"] == int(g["seed_n_supersonic"])
    assert st["n_term3_active"] == int(g["n_term3_active"])
    J_ff, B = sysm.blocks(st)
    n_f = len(g["free"])
    J_ref = sp.csr_matrix((g["Jff_data"], g["Jff_indices"], g["Jff_indptr"]), shape=(n_f, n_f))
    assert _rel(J_ff.toarray(), J_ref.toarray()) <= 1e-12
    assert _rel(B.toarray(), g["B"]) <= 1e-12
    y = J_ff @ g["x"] + B @ (sysm.K @ g["x"])
    assert _rel(y, g["y"]) <= 1e-12
    assert _rel(B @ F, g["BF"]) <= 1e-12


@pytest.mark.parametrize("name", CASES)
def test_oracle_lifting_solve_matches_reference(gold, name):
    from up3d_b200.constraints.dirichlet import freestream_phi
    g, cut = _case(gold, name)
    sysm = _system(g, cut)
    phi0 = freestream_phi(g["nodes"][:sysm.n_red], float(g["alpha_deg"]), 1.0)
    phi, gamma, hist, ok = sysm.solve(phi0[sysm.free], np.zeros(sysm.n_st), float(g["m_inf"]))
    assert ok
    assert len(hist) - 1 == int(g["sol_n_newton"])
    assert np.max(np.abs(phi - g["sol_phi"])) <= 1e-10
    assert np.max(np.abs(gamma - g["sol_gamma"])) <= 1e-10


def test_oracle_lifting_taper_and_external_rhs_match_reference(gold):
    """A tapered Kutta row and a lagged external right-hand side
    (solve/newton.py:165-214, :399-419): the reference's converged solution."""
    from up3d_b200.constraints.dirichlet import freestream_phi
    from oracle import oracle as O
    g, cut = _case(gold, "sub")
    sysm = O.LiftingSystem(g["nodes"], g["elements"], cut.wc, g["dir_red"], g["vals0_red"], g["V_red"],
                           tip_taper=g["taper"], external_rhs=g["external_rhs"])
    phi0 = freestream_phi(g["nodes"][:sysm.n_red], float(g["alpha_deg"]), 1.0)
    phi, gamma, hist, ok = sysm.solve(phi0[sysm.free], np.zeros(sysm.n_st), float(g["m_inf"]))
    assert ok and len(hist) - 1 == int(g["taper_n_newton"])
    assert np.max(np.abs(phi - g["taper_phi"])) <= 1e-10
    assert np.max(np.abs(gamma - g["taper_gamma"])) <= 1e-10


def test_lifting_drivers_at_the_reference_module_paths():
    """The reference keeps the coupled workspace and drivers in
    solve/newton.py and the lifting Picard in solve/picard.py: the same
    imports work here."""
    from up3d_b200.solve import lifting
    from up3d_b200.solve.newton import NewtonWorkspace, solve_newton_lifting, solve_newton_transonic
    from up3d_b200.solve.picard import solve_subsonic_lifting
    assert NewtonWorkspace is lifting.NewtonWorkspace
    assert solve_newton_lifting is lifting.solve_newton_lifting
    assert solve_subsonic_lifting is lifting.solve_subsonic_lifting
    assert callable(solve_newton_transonic)
