"""Parity of the CUDA hot path (through the C ABI) with the reference's golden
fixtures and with the CPU oracle, on identical meshes and inputs.

Bar: FP64 results within REL_TOL = 1e-12 of max|reference| (summation order
and libm rounding differ); integer outputs (walk, branches, pattern, maps)
exact.  Mirrors the reference's hot-path tests (tests/test_p3_assembly.py,
test_p4_upwind.py, test_p7_diff_flux.py, test_p8_jacobian.py).
"""

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import REL_TOL, has_cuda, rel_err, sparse_rel_err
from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]

M_CRIT, UPWIND_C, RHO_FLOOR, M_CAP = 0.95, 1.5, 0.05, 3.0
LABELS = ["freestream_m05", "seed0_m085", "accelerating_m08", "shockpoint_m08", "mixed_m08",
          "limited_m08"]


@pytest.fixture(scope="module")
def gpu_small(small_golden):
    from up3d_b200.kernels.jacobian import PicardOperator
    from up3d_b200.kernels.upwind import UpwindOperator
    g = small_golden
    return PicardOperator(g.mesh("nodes"), g.mesh("elements")), UpwindOperator(g.mesh("nodes"), g.mesh("elements"))


@pytest.fixture(scope="module")
def oracle_small(small_golden):
    g = small_golden
    return O.PicardOperator(g.mesh("nodes"), g.mesh("elements")), O.UpwindOperator(g.mesh("nodes"), g.mesh("elements"))


def _gpu_chain(op, upw, phi, m):
    """eval_residual + assemble_coupled through the drop-in API
    (pyfp3d/solve/newton.py:345-372, :435-452)."""
    from up3d_b200.physics.isentropic import density_field, limit_q2_field
    out = {}
    grad, q2 = op.velocities(phi)
    grad, q2 = grad.copy(), q2.copy()
    q2l = limit_q2_field(q2, m, M_CAP)
    lim = q2l == q2
    rho = density_field(q2l, m)
    rt = upw.rho_tilde(grad, q2l, rho, m, UPWIND_C, M_CRIT, rho_floor=RHO_FLOOR).copy()
    out.update(grad=grad, q2=q2, q2l=q2l, lim=lim, rho=rho, rho_tilde=rt, nu=upw.nu.copy(),
               upstream=upw._upstream.copy(), nu_max=upw.nu_max, n_supersonic=upw.n_supersonic,
               n_floored=upw.n_floored)
    up, br = upw.freeze_upwind_state(grad, q2l, rho, m, UPWIND_C, M_CRIT, rho_floor=RHO_FLOOR)
    out["branch"] = br
    out["rho_tilde_frozen"] = upw.rho_tilde_frozen(q2l, rho, up, br, m, UPWIND_C, M_CRIT,
                                                   rho_floor=RHO_FLOOR).copy()
    se_f, su_f = upw.rho_tilde_frozen_sensitivities(q2l, rho, up, br, m, UPWIND_C, M_CRIT,
                                                    rho_floor=RHO_FLOOR)
    out.update(s_e_frozen=se_f.copy(), s_u_frozen=su_f.copy())
    s_e, s_u, upstream = upw.rho_tilde_sensitivities(grad, q2l, rho, m, UPWIND_C, M_CRIT,
                                                     rho_floor=RHO_FLOOR)
    s_e, s_u, upstream = s_e.copy(), s_u.copy(), upstream.copy()
    out.update(s_e=s_e, s_u=s_u)
    out["R"] = op.assemble_residual(phi, rt).copy()
    out["A"] = op.assemble_matrix(rt)
    out["J"] = op.assemble_newton_jacobian(phi, rt, s_e, s_u, upstream,
                                           lim_mask=None if lim.all() else lim)
    out["n_term3_active"] = op.n_term3_active
    out["newton_nnz"] = op.newton_nnz
    return out


def test_mesh_setup_matches_reference(gpu_small, small_golden):
    op, upw = gpu_small
    g = small_golden
    assert rel_err(op.B, g.mesh("B")) < 1e-14
    assert rel_err(op.V, g.mesh("V")) < 1e-14
    assert np.array_equal(upw.face_neighbors, g.mesh("face_neighbors"))
    assert np.array_equal(upw.centroids, g.mesh("centroids"))
    assert np.array_equal(op.color_offsets, g.mesh("color_offsets"))
    assert np.array_equal(op.color_elems, g.mesh("color_elems"))
    assert np.array_equal(op._pattern.indptr, g.mesh("indptr"))
    assert np.array_equal(op._pattern.indices, g.mesh("indices"))
    assert np.array_equal(op.elem_to_csr, g.mesh("elem_to_csr"))
    assert rel_err(op.assemble_matrix().data, g.mesh("laplace_data")) < REL_TOL


def test_geometry_bitwise_equals_oracle(gpu_small, oracle_small):
    op, upw = gpu_small
    oop, oupw = oracle_small
    assert np.array_equal(op.B, oop.B)
    assert np.array_equal(op.V, oop.V)


@pytest.mark.parametrize("label", LABELS)
def test_api_chain_matches_reference(gpu_small, oracle_small, small_golden, label):
    op, upw = gpu_small
    g = small_golden
    phi, m = g.state(label, "phi"), float(g.state(label, "m_inf"))
    r = _gpu_chain(op, upw, phi, m)
    for key in ("q2", "q2l", "rho", "rho_tilde", "nu", "s_e", "s_u", "R", "rho_tilde_frozen",
                "s_e_frozen", "s_u_frozen"):
        assert rel_err(r[key], g.state(label, key)) < REL_TOL, key
    assert np.array_equal(r["lim"], g.state(label, "lim"))
    assert np.array_equal(r["branch"], g.state(label, "branch"))
    # the walk, the limiter and the switch are IEEE-exact: identical to the oracle
    oop, oupw = oracle_small
    ro = O.chain(oop, oupw, phi, m)
    assert np.array_equal(r["grad"], ro["grad"])
    assert np.array_equal(r["q2"], ro["q2"])
    assert np.array_equal(r["upstream"], ro["upstream"])
    assert np.array_equal(r["nu"], ro["nu"]) or np.all(r["nu"] == 0)
    if not label.startswith("freestream"):
        assert np.array_equal(r["upstream"], g.state(label, "upstream"))
    assert r["n_supersonic"] == int(g.state(label, "n_supersonic"))
    assert r["n_floored"] == int(g.state(label, "n_floored"))
    assert r["nu_max"] == pytest.approx(float(g.state(label, "nu_max")), rel=1e-13)
    assert rel_err(r["A"].data, g.state(label, "A_data")) < REL_TOL
    Jg = sp.csr_matrix((g.state(label, "J_data"), g.state(label, "J_indices"),
                        g.state(label, "J_indptr")), shape=r["J"].shape)
    assert sparse_rel_err(r["J"], Jg) < REL_TOL
    assert r["n_term3_active"] == int(g.state(label, "n_term3_active"))
    tiny = np.count_nonzero(np.abs(Jg.data) < 1e-14 * np.abs(Jg.data).max())
    assert Jg.nnz - tiny <= r["newton_nnz"] <= Jg.nnz
    assert r["J"].nnz == r["newton_nnz"]


@pytest.mark.parametrize("label", LABELS)
def test_fused_matches_reference(small_golden, label):
    import torch
    from up3d_b200.mesh.device import get_mesh
    from up3d_b200.solve.fused import FlowParams, ResidualJacobian
    g = small_golden
    mesh = get_mesh(g.mesh("nodes"), g.mesh("elements"))
    ev = ResidualJacobian(mesh)
    phi = torch.from_numpy(g.state(label, "phi")).cuda()
    ev.evaluate(phi, FlowParams(m_inf=float(g.state(label, "m_inf"))))
    assert rel_err(ev.R.cpu().numpy(), g.state(label, "R")) < REL_TOL
    assert rel_err(ev.rho_tilde.cpu().numpy(), g.state(label, "rho_tilde")) < REL_TOL
    if not label.startswith("freestream"):
        assert np.array_equal(ev.upstream.cpu().numpy(), g.state(label, "upstream"))
    mon = ev.read_monitors()
    assert mon["n_supersonic"] == int(g.state(label, "n_supersonic"))
    assert mon["n_floored"] == int(g.state(label, "n_floored"))
    assert mon["n_limited"] == int((~g.state(label, "lim")).sum())
    assert mon["n_term3_active"] == int(g.state(label, "n_term3_active"))
    J = ev.jacobian().to_scipy()
    Jg = sp.csr_matrix((g.state(label, "J_data"), g.state(label, "J_indices"),
                        g.state(label, "J_indptr")), shape=J.shape)
    assert sparse_rel_err(J, Jg) < REL_TOL


@pytest.mark.parametrize("label", ["seed0_m05", "mixed_m08"])
def test_c1_matches_reference(c1_golden, label):
    import torch
    from up3d_b200.kernels.jacobian import PicardOperator
    from up3d_b200.mesh.device import get_mesh
    from up3d_b200.solve.fused import FlowParams, ResidualJacobian
    g = c1_golden
    mesh = get_mesh(g.mesh("nodes"), g.mesh("elements"))
    ev = ResidualJacobian(mesh)
    phi = torch.from_numpy(g.state(label, "phi")).cuda()
    ev.evaluate(phi, FlowParams(m_inf=float(g.state(label, "m_inf"))))
    for key, dev in (("R", ev.R), ("rho_tilde", ev.rho_tilde)):
        assert rel_err(dev.cpu().numpy(), g.state(label, key)) < REL_TOL, key
    assert np.array_equal(ev.upstream.cpu().numpy(), g.state(label, "upstream"))
    J = ev.jacobian().to_scipy()
    Jg = sp.csr_matrix((g.state(label, "J_data"), g.state(label, "J_indices"),
                        g.state(label, "J_indptr")), shape=J.shape)
    assert sparse_rel_err(J, Jg) < REL_TOL
    op = PicardOperator(g.mesh("nodes"), g.mesh("elements"))
    assert rel_err(op.assemble_matrix(g.state(label, "rho_tilde")).data, g.state(label, "A_data")) < REL_TOL
    assert np.array_equal(op.color_offsets, g.mesh("color_offsets"))


def test_fused_is_bit_reproducible(small_golden):
    import torch
    from up3d_b200.mesh.device import get_mesh
    from up3d_b200.solve.fused import FlowParams, ResidualJacobian
    g = small_golden
    ev = ResidualJacobian(get_mesh(g.mesh("nodes"), g.mesh("elements")))
    phi = torch.from_numpy(g.state("mixed_m08", "phi")).cuda()
    ev.evaluate(phi, FlowParams(m_inf=0.8))
    R1, J1 = ev.R.clone(), ev.jacobian().to_scipy()
    ev.evaluate(phi, FlowParams(m_inf=0.8))
    R2, J2 = ev.R.clone(), ev.jacobian().to_scipy()
    assert torch.equal(R1, R2)
    assert np.array_equal(J1.data, J2.data) and np.array_equal(J1.indices, J2.indices)


def test_jacobian_reduces_to_picard_bitwise(gpu_small, small_golden):
    """J == A bitwise at s = 0 (reference tests/test_p8_jacobian.py:242-244)."""
    op, upw = gpu_small
    phi = small_golden.state("seed0_m085", "phi")
    rt = small_golden.state("seed0_m085", "rho_tilde")
    z = np.zeros(op.n_tets)
    J0 = op.assemble_newton_jacobian(phi, rt, z, z, np.arange(op.n_tets))
    A = op.assemble_matrix(rt)
    assert op.n_term3_active == 0
    assert np.array_equal(J0.indptr, A.indptr) and np.array_equal(J0.indices, A.indices)
    assert np.array_equal(J0.data, A.data)


def test_limiter_mask_gates_the_chain(gpu_small, small_golden):
    """reference tests/test_p8_jacobian.py:247-271"""
    op, upw = gpu_small
    label = "accelerating_m08"
    g = small_golden
    phi, rt = g.state(label, "phi"), g.state(label, "rho_tilde")
    s_e, s_u = g.state(label, "s_e").copy(), g.state(label, "s_u").copy()
    up = g.state(label, "upstream")
    se0, su0 = s_e.copy(), s_u.copy()
    J = op.assemble_newton_jacobian(phi, rt, s_e, s_u, up, lim_mask=np.zeros(op.n_tets, dtype=bool))
    A = op.assemble_matrix(rt)
    assert op.n_term3_active == 0
    assert np.array_equal(J.data, A.data)
    assert np.array_equal(s_e, se0) and np.array_equal(s_u, su0)


def test_frozen_equals_live_at_freeze(gpu_small, small_golden):
    """reference tests/test_p8_jacobian.py:277-302"""
    from up3d_b200.physics.isentropic import density_field
    op, upw = gpu_small
    phi = small_golden.state("mixed_m08", "phi")
    grad, q2 = op.velocities(phi)
    grad, q2 = grad.copy(), q2.copy()
    rho = density_field(q2, 0.8)
    live = upw.rho_tilde(grad, q2, rho, 0.8, UPWIND_C, M_CRIT).copy()
    up, br = upw.freeze_upwind_state(grad, q2, rho, 0.8, UPWIND_C, M_CRIT)
    frozen = upw.rho_tilde_frozen(q2, rho, up, br, 0.8, UPWIND_C, M_CRIT).copy()
    assert np.array_equal(live, frozen)
    assert (br == 1).sum() > 0 and (br == 2).sum() > 0


def test_forward_paths_untouched_by_jacobian(gpu_small, small_golden):
    """reference tests/test_p8_jacobian.py:361-389"""
    op, upw = gpu_small
    g = small_golden
    label = "mixed_m08"
    phi, rt = g.state(label, "phi"), g.state(label, "rho_tilde")
    A_ref = op.assemble_matrix(rt).data.copy()
    R_ref = op.assemble_residual(phi, rt).copy()
    op.assemble_newton_jacobian(phi, rt, g.state(label, "s_e"), g.state(label, "s_u"),
                                g.state(label, "upstream"))
    assert np.array_equal(A_ref, op.assemble_matrix(rt).data)
    assert np.array_equal(R_ref, op.assemble_residual(phi, rt))


def test_device_tensors_in_device_tensors_out(gpu_small, small_golden):
    import torch
    from up3d_b200.mesh.device import DeviceCSR
    op, upw = gpu_small
    phi = torch.from_numpy(small_golden.state("seed0_m085", "phi")).cuda()
    grad, q2 = op.velocities(phi)
    assert grad.is_cuda and q2.is_cuda
    R = op.assemble_residual(phi)
    assert R.is_cuda
    A = op.assemble_matrix(torch.ones(op.n_tets, dtype=torch.float64, device="cuda"))
    assert isinstance(A, DeviceCSR)
    assert rel_err(A.data.cpu().numpy(), small_golden.mesh("laplace_data")) < REL_TOL


def test_spmv_matches_scipy(small_golden):
    import torch
    from up3d_b200.kernels.jacobian import PicardOperator
    g = small_golden
    op = PicardOperator(torch.from_numpy(g.mesh("nodes")), torch.from_numpy(g.mesh("elements")))
    A = op.assemble_matrix(torch.ones(op.n_tets, dtype=torch.float64, device="cuda"))
    x = torch.linspace(-1.0, 2.0, op.n_nodes, dtype=torch.float64, device="cuda")
    y = A.matvec(x).cpu().numpy()
    ref = A.to_scipy() @ x.cpu().numpy()
    assert rel_err(y, ref) < 1e-14
    dirichlet = torch.zeros(op.n_nodes, dtype=torch.uint8, device="cuda")
    dirichlet[g.mesh("dirichlet_nodes")] = 1
    yd = A.matvec(x, dirichlet=dirichlet).cpu().numpy()
    As = A.to_scipy()
    free = np.setdiff1d(np.arange(op.n_nodes), g.mesh("dirichlet_nodes"))
    xf = x.cpu().numpy()
    assert rel_err(yd[free], As[free][:, free] @ xf[free]) < 1e-14
    assert np.array_equal(yd[g.mesh("dirichlet_nodes")], xf[g.mesh("dirichlet_nodes")])


def test_degenerate_tet_raises():
    from up3d_b200.kernels.jacobian import PicardOperator
    nodes = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0.0]])
    with pytest.raises(ValueError, match="degenerate"):
        PicardOperator(nodes, np.array([[0, 1, 2, 3]], dtype=np.int32))


def test_out_of_range_connectivity_raises():
    from up3d_b200.kernels.jacobian import PicardOperator
    nodes = np.eye(4, 3)
    with pytest.raises(ValueError, match="out of range"):
        PicardOperator(nodes, np.array([[0, 1, 2, 7]], dtype=np.int32))
