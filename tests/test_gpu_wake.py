"""The wake master-slave elimination on the device (constraints/wake.py:
32-212) against the reference's WakeConstraint / kutta_targets
(tests/golden/wake_constraint.npz) and the oracle, host and device inputs."""

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN, has_cuda

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "wake_constraint.npz")


def _cut(single, shape=(10, 4, 4)):
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.mesh.wake_cut import cut_channel_sheet
    return cut_channel_sheet(bump_channel(*shape, amplitude=0.08, seed=1), single_station=single)


def _csr(g, q, n_rows, n_cols):
    return sp.csr_matrix((g[q + "data"], g[q + "indices"], g[q + "indptr"]), shape=(n_rows, n_cols))


def _close(a, b, scale, tol=1e-14):
    return np.abs(np.asarray(a) - np.asarray(b)).max() <= tol * scale


def _same_matrix(ours, ref, scale, tol=1e-14):
    """Equal values.  The reference's scipy products drop entries that sum
    to exactly zero (the Kuhn channel's right-angle edges have zero
    stiffness); the device keeps the structural pattern, so it may hold
    extra explicit zeros and nothing else."""
    D = (sp.csr_matrix(ours) - sp.csr_matrix(ref)).tocoo()
    return not D.nnz or np.abs(D.data).max() <= tol * scale


@pytest.mark.parametrize("tag", ["multi", "single"])
@pytest.mark.parametrize("mat", ["picard", "newton"])
def test_wake_constraint_matches_reference(gold, tag, mat):
    from up3d_b200.constraints.wake import WakeConstraint, kutta_targets
    cut = _cut(tag == "single")
    q = f"{tag}/{mat}/"
    n_cut = len(cut.nodes)
    A = _csr(gold, q + "A_", n_cut, n_cut)
    con = WakeConstraint(A, cut.wc)
    n_red, n_st = con.n_reduced, cut.wc.n_stations
    ref_red, ref_H = _csr(gold, q + "red_", n_red, n_red), _csr(gold, q + "H_", n_red, n_st)
    scale = np.abs(ref_red.data).max()
    A_red, H = con.reduce_operator(A)
    assert isinstance(A_red, sp.csr_matrix)
    assert A_red.nnz >= ref_red.nnz and H.nnz >= ref_H.nnz
    assert _same_matrix(A_red, ref_red, scale) and _same_matrix(H, ref_H, scale)
    assert _same_matrix(con.A_reduced, ref_red, scale)
    assert _close(con._h, gold[q + "h_dense"], scale)
    rhs = con.reduced_rhs(gold[q + "b"], gold[q + "gamma"])
    assert _close(rhs, gold[q + "rhs"], np.abs(gold[q + "rhs"]).max(), 1e-13)
    assert np.array_equal(con.expand(gold[q + "phi_red"], gold[q + "gamma"]), gold[q + "expand"])
    dn, dv = con.to_reduced_dirichlet(cut.dirichlet_nodes, gold[f"{tag}/dir_values"])
    assert np.array_equal(dn, gold[f"{tag}/red_dir_nodes"]) and np.array_equal(dv, gold[f"{tag}/red_dir_values"])
    assert _close(kutta_targets(gold[f"{tag}/phi_cut"], cut.wc), gold[f"{tag}/kutta"], 1.0, 1e-15)


def test_device_inputs_match_host_inputs_bitwise(gold):
    import torch
    from up3d_b200.constraints.wake import WakeConstraint, kutta_targets
    from up3d_b200.mesh.device import DeviceCSR
    cut = _cut(False)
    q = "multi/newton/"
    n_cut = len(cut.nodes)
    A = _csr(gold, q + "A_", n_cut, n_cut)
    dA = DeviceCSR(torch.from_numpy(A.indptr.astype(np.int32)).cuda(), torch.from_numpy(A.indices).cuda(),
                   torch.from_numpy(A.data).cuda(), A.shape)
    host = WakeConstraint(A, cut.wc)
    dev = WakeConstraint(dA, cut.wc)
    R_h, H_h = host.reduce_operator(A)
    R_d, H_d = dev.reduce_operator(dA)
    assert (R_d.to_scipy() != R_h).nnz == 0 and (H_d.to_scipy() != H_h).nnz == 0
    b, g = torch.from_numpy(gold[q + "b"]).cuda(), torch.from_numpy(gold[q + "gamma"]).cuda()
    assert np.array_equal(dev.reduced_rhs(b, g).cpu().numpy(), host.reduced_rhs(gold[q + "b"], gold[q + "gamma"]))
    p = torch.from_numpy(gold[q + "phi_red"]).cuda()
    assert np.array_equal(dev.expand(p, g).cpu().numpy(), gold[q + "expand"])
    k = kutta_targets(torch.from_numpy(gold["multi/phi_cut"]).cuda(), cut.wc)
    assert np.abs(k.cpu().numpy() - gold["multi/kutta"]).max() <= 1e-15


def test_newton_jacobian_of_a_larger_cut_matches_the_oracle():
    """The device Newton Jacobian of a cut channel (P1 pattern plus the
    Term-3 entries) reduced on the device, against the oracle's scipy
    reduction of the same matrix; the same constraint first serves the
    Picard pattern, then the Newton one."""
    import torch
    from oracle import oracle as O
    from up3d_b200.constraints.wake import WakeConstraint
    from up3d_b200.mesh.device import DeviceMesh
    from up3d_b200.mesh.kuhn import bump_channel, pocket_state
    from up3d_b200.solve.fused import FlowParams, ResidualJacobian
    mesh = bump_channel(40, 10, 10, amplitude=0.08, seed=3)
    from up3d_b200.mesh.wake_cut import cut_channel_sheet
    cut = cut_channel_sheet(mesh)
    wc = cut.wc
    phi0 = pocket_state(mesh, "mixed")
    phi = np.concatenate([phi0, phi0[wc.master_nodes] + 0.02])
    dm = DeviceMesh(cut.nodes, cut.elements)
    ev = ResidualJacobian(dm)
    ev.evaluate(torch.from_numpy(phi).cuda(), FlowParams(m_inf=0.8), jacobian=True)
    assert ev.read_monitors()["n_term3_active"] > 0
    A_p = ev.jacobian()                     # merged CSR: P1 pattern + Term-3 extras
    lap = dm.indptr, dm.indices
    from up3d_b200.mesh.device import DeviceCSR
    P = DeviceCSR(lap[0], lap[1], torch.rand(dm.nnz, dtype=torch.float64, device="cuda"), A_p.shape)
    con = WakeConstraint(P, wc)
    for M in (P, A_p, P):
        ref = O.WakeConstraint(M.to_scipy(), wc)
        R, H = con.reduce_operator(M)
        R, H = R.to_scipy(), H.to_scipy()
        scale = np.abs(ref.A_reduced.data).max()
        assert _same_matrix(R, ref.A_reduced, scale)
        assert np.abs(H.toarray() - ref._h.T).max() <= 1e-14 * scale
    assert len(con._plans) == 2             # two patterns, each planned once


def test_size_mismatch_raises():
    from up3d_b200.constraints.wake import WakeConstraint
    cut = _cut(False)
    A = sp.identity(len(cut.nodes) - 1, format="csr")
    with pytest.raises(ValueError, match="WakeCut implies"):
        WakeConstraint(A, cut.wc)
