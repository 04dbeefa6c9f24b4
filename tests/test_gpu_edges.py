"""Edge cases of the hot path on the device, against the oracle: a single
tet, disconnected tets, a node that belongs to no element, a mesh with no
supersonic element, and the empty inputs of the wake elimination and the
wall post-processing."""

import numpy as np
import pytest

from conftest import has_cuda, rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]


def _evaluate(nodes, elements, phi, m_inf):
    import torch
    from up3d_b200.mesh.device import DeviceMesh
    from up3d_b200.solve.fused import FlowParams, ResidualJacobian
    dm = DeviceMesh(nodes, elements)
    ev = ResidualJacobian(dm)
    R = ev.evaluate(torch.from_numpy(phi).cuda(), FlowParams(m_inf=m_inf), jacobian=True).cpu().numpy()
    return R, ev.jacobian().to_scipy(), ev.read_monitors()


def _oracle(nodes, elements, phi, m_inf):
    from oracle import oracle as O
    return O.chain(O.PicardOperator(nodes, elements), O.UpwindOperator(nodes, elements), phi, m_inf)


def _check(nodes, elements, phi, m_inf):
    R, J, mon = _evaluate(nodes, elements, phi, m_inf)
    ref = _oracle(nodes, elements, phi, m_inf)
    assert rel_err(R, ref["R"]) < 1e-12
    D = (J - ref["J"]).tocoo()
    assert (np.abs(D.data).max() if D.nnz else 0.0) <= 1e-12 * max(np.abs(ref["J"].data).max(), 1e-300)
    assert mon["n_term3_active"] == ref["n_term3_active"]
    return R, J, ref


def test_single_tet():
    nodes = np.array([[0.0, 0.0, 0.0], [1.0, 0.1, 0.0], [0.2, 1.0, 0.1], [0.1, 0.2, 0.9]])
    el = np.array([[0, 1, 2, 3]], dtype=np.int32)
    for phi in (nodes[:, 0].copy(), np.array([0.0, 1.6, 0.3, -0.2])):
        R, J, _ = _check(nodes, el, phi, 0.8)
        assert J.shape == (4, 4) and J.nnz == 16


def test_disconnected_tets_and_an_isolated_node():
    nodes = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0],
                      [3.0, 0.0, 0.0], [4.0, 0.1, 0.0], [3.1, 1.0, 0.0], [3.0, 0.2, 1.1],
                      [9.0, 9.0, 9.0]])                    # node 8: in no element
    el = np.array([[0, 1, 2, 3], [4, 5, 6, 7]], dtype=np.int32)
    phi = np.array([0.0, 1.2, 0.1, 0.0, 3.0, 4.4, 3.2, 3.0, 7.0])
    R, J, ref = _check(nodes, el, phi, 0.7)
    assert R[8] == 0.0 and J.indptr[9] == J.indptr[8]          # empty row
    # the same two tets without the isolated node: the same numbers
    R2, J2, _ = _check(nodes[:8], el, phi[:8], 0.7)
    assert np.array_equal(R[:8], R2) and (J[:8, :8] != J2).nnz == 0


def test_all_subsonic_state_has_no_term3():
    from up3d_b200.mesh.kuhn import bump_channel
    m = bump_channel(8, 3, 3, amplitude=0.02, seed=4)
    R, J, ref = _check(m.nodes, m.elements, m.freestream(), 0.5)
    assert ref["n_term3_active"] == 0


def test_wake_without_slaves_is_the_identity_fold():
    import scipy.sparse as sp
    from up3d_b200.constraints.wake import WakeConstraint
    from up3d_b200.mesh.wake_cut import WakeCut
    A = sp.random(30, 30, density=0.2, random_state=np.random.default_rng(2), format="csr")
    A.sort_indices()
    con = WakeConstraint(A, WakeCut(n_nodes_orig=30))
    R, H = con.reduce_operator(A)
    assert (R != A).nnz == 0 and H.shape == (30, 0)
    b = np.arange(30.0)
    assert np.array_equal(con.reduced_rhs(b, np.zeros(0)), b)
    assert np.array_equal(con.expand(b, np.zeros(0)), b)


def test_wall_without_faces_gives_zero_force():
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.post.surface import wall_force_coefficients
    m = bump_channel(6, 3, 3, amplitude=0.0, seed=0)
    r = wall_force_coefficients(m.nodes, m.elements, np.zeros((0, 3), dtype=np.int64), m.freestream())
    assert np.array_equal(r["cf"], np.zeros(3)) and r["cl"] == 0.0 and len(r["cp_tri"]) == 0
