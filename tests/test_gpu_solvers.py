"""Device Krylov solvers and the AMG preconditioner against scipy's direct
solve of the same reduced systems (the reference solves them with
spla.cg / spla.gmres + pyamg, solve/linear.py:134-239)."""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from conftest import has_cuda, rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def c1_system(c1_golden):
    """Picard matrix and Newton Jacobian of the C1 mesh at the mixed state,
    on device and as scipy, with the inflow/outflow Dirichlet split."""
    import torch
    from up3d_b200.kernels.jacobian import PicardOperator
    g = c1_golden
    op = PicardOperator(g.mesh("nodes"), g.mesh("elements"))
    label = "mixed_m08"
    rt = torch.from_numpy(g.state(label, "rho_tilde")).cuda()
    A = op.assemble_matrix(rt)
    phi = torch.from_numpy(g.state(label, "phi")).cuda()
    J = op.assemble_newton_jacobian(phi, rt, torch.from_numpy(g.state(label, "s_e")).cuda(),
                                    torch.from_numpy(g.state(label, "s_u")).cuda(),
                                    torch.from_numpy(g.state(label, "upstream").astype(np.int64)).cuda())
    dn = g.mesh("dirichlet_nodes")
    n = op.n_nodes
    free = np.setdiff1d(np.arange(n), dn)
    mask = torch.zeros(n, dtype=torch.uint8, device="cuda")
    mask[torch.from_numpy(dn).cuda()] = 1
    rng = np.random.default_rng(5)
    b = rng.standard_normal(n)
    b[dn] = 0.0
    return {"A": A, "J": J, "mask": mask, "free": free, "b": b, "n": n}


def _embedded(M, mask):
    from up3d_b200.solve.linear import with_dirichlet
    return with_dirichlet(M, mask)


def _direct(M, free, b):
    Ms = M.to_scipy()
    x = np.zeros(len(b))
    x[free] = spla.spsolve(Ms[free][:, free].tocsc(), b[free])
    return x


def test_cg_jacobi_matches_direct(c1_system):
    import torch
    from up3d_b200.solve.linear import build_jacobi_preconditioner, solve_cg
    s = c1_system
    A = _embedded(s["A"], s["mask"])
    M = build_jacobi_preconditioner(A)
    x, it, info = solve_cg(A, torch.from_numpy(s["b"]).cuda(), M=M, rtol=1e-12, maxiter=5000)
    assert info == 0
    ref = _direct(s["A"], s["free"], s["b"])
    assert rel_err(x.cpu().numpy(), ref) < 1e-9


@pytest.mark.parametrize("fp32", [False, True])
def test_cg_amg_matches_direct(c1_system, fp32):
    import torch
    from up3d_b200.solve.linear import build_amg_preconditioner, build_jacobi_preconditioner, solve_cg
    s = c1_system
    A = _embedded(s["A"], s["mask"])
    ml, M = build_amg_preconditioner(A, fp32=fp32)
    assert ml.n_levels >= 2 and ml.operator_complexity < 3.0
    b = torch.from_numpy(s["b"]).cuda()
    x, it_amg, info = solve_cg(A, b, M=M, rtol=1e-12, maxiter=500)
    assert info == 0
    ref = _direct(s["A"], s["free"], s["b"])
    assert rel_err(x.cpu().numpy(), ref) < 1e-9
    _, it_jac, _ = solve_cg(A, b, M=build_jacobi_preconditioner(A), rtol=1e-12, maxiter=5000)
    assert it_amg < it_jac / 3, (it_amg, it_jac)


def test_amg_setup_is_deterministic(c1_system):
    import torch
    from up3d_b200.solve.linear import build_amg_preconditioner
    s = c1_system
    A = _embedded(s["A"], s["mask"])
    r = torch.from_numpy(s["b"]).cuda()
    z1 = build_amg_preconditioner(A)[1].matvec(r)
    z2 = build_amg_preconditioner(A)[1].matvec(r)
    assert torch.equal(z1, z2)


@pytest.mark.parametrize("fp32", [False, True])
def test_amg_refresh_equals_fresh_setup(c1_system, fp32):
    """A hierarchy set up on one Picard matrix and refreshed with another of
    the same pattern applies bit-identically to a fresh setup on the second
    (the aggregates depend on the pattern only)."""
    import torch
    from up3d_b200.kernels.jacobian import PicardOperator
    from up3d_b200.solve.linear import build_amg_preconditioner
    s = c1_system
    A2 = _embedded(s["A"], s["mask"])
    rng = np.random.default_rng(9)
    A1 = _embedded(s["A"], s["mask"])
    A1.data = A1.data * torch.from_numpy(1.0 + 0.5 * rng.random(A1.data.numel())).cuda()
    r = torch.from_numpy(s["b"]).cuda()
    _, M = build_amg_preconditioner(A1, fp32=fp32)
    z1 = M.matvec(r)
    M.refresh(A2)
    z_ref = build_amg_preconditioner(A2, fp32=fp32)[1].matvec(r)
    assert torch.equal(M.matvec(r), z_ref)
    assert not torch.equal(z1, z_ref)


def test_amg_refresh_rejects_another_pattern(c1_system):
    import torch
    from up3d_b200.solve.linear import build_amg_preconditioner, with_dirichlet
    s = c1_system
    _, M = build_amg_preconditioner(_embedded(s["A"], s["mask"]))
    other = s["mask"].clone()
    other[int(s["free"][0])] = 1
    with pytest.raises(ValueError, match="pattern|mask"):
        M.refresh(with_dirichlet(s["A"], other))
    with pytest.raises(ValueError, match="pattern|mask"):
        M.refresh(s["A"])


def test_gmres_amg_on_newton_jacobian(c1_system):
    import torch
    from up3d_b200.solve.linear import build_amg_preconditioner, solve_gmres, with_dirichlet
    s = c1_system
    J = with_dirichlet(s["J"], s["mask"])
    A = with_dirichlet(s["A"], s["mask"])
    _, M = build_amg_preconditioner(A)
    b = torch.from_numpy(s["b"]).cuda()
    x, n_inner, info = solve_gmres(J, b, M=M, rtol=1e-11, restart=60, maxiter=20)
    assert info == 0
    ref = _direct(s["J"], s["free"], s["b"])
    assert rel_err(x.cpu().numpy(), ref) < 1e-8
    assert n_inner > 0


def test_solve_gmres_scipy_inputs_return_numpy(c1_system):
    from up3d_b200.solve.linear import solve_gmres
    s = c1_system
    free = s["free"]
    Js = s["J"].to_scipy()[free][:, free].tocsr()
    b = s["b"][free]
    x, n_inner, info = solve_gmres(Js, b, rtol=1e-10, restart=200, maxiter=50, on_fail="return")
    assert isinstance(x, np.ndarray)
    r = np.linalg.norm(Js @ x - b) / np.linalg.norm(b)
    assert (info == 0 and r < 1e-9) or info != 0


def test_cg_amg_drop_in(c1_system):
    from up3d_b200.solve.linear import solve_cg_amg
    s = c1_system
    free = s["free"]
    As = s["A"].to_scipy()[free][:, free].tocsr()
    b = s["b"][free]
    x, n_it = solve_cg_amg(As, b, rtol=1e-10)
    assert isinstance(x, np.ndarray)
    assert np.linalg.norm(As @ x - b) <= 1e-10 * np.linalg.norm(b) * 1.01


def test_gmres_mixed_refines_to_fp64_accuracy(c1_golden):
    """FP32 inner GMRES (FP32 Jacobian values, FP32 AMG) with FP64 refinement
    reaches the FP64 direct solution of the C1 Newton system at the
    subsonic seeded state; one FP32 solve alone does not."""
    import torch
    from up3d_b200.kernels.jacobian import PicardOperator
    from up3d_b200.solve.linear import build_amg_preconditioner, solve_gmres_mixed, with_dirichlet
    g = c1_golden
    op = PicardOperator(g.mesh("nodes"), g.mesh("elements"))
    label = "seed0_m05"
    rt = torch.from_numpy(g.state(label, "rho_tilde")).cuda()
    phi = torch.from_numpy(g.state(label, "phi")).cuda()
    J = op.assemble_newton_jacobian(phi, rt, torch.from_numpy(g.state(label, "s_e")).cuda(),
                                    torch.from_numpy(g.state(label, "s_u")).cuda(),
                                    torch.from_numpy(g.state(label, "upstream").astype(np.int64)).cuda())
    dn = g.mesh("dirichlet_nodes")
    n = op.n_nodes
    free = np.setdiff1d(np.arange(n), dn)
    mask = torch.zeros(n, dtype=torch.uint8, device="cuda")
    mask[torch.from_numpy(dn).cuda()] = 1
    b = np.random.default_rng(5).standard_normal(n)
    b[dn] = 0.0
    _, M = build_amg_preconditioner(with_dirichlet(op.assemble_matrix(rt), mask), fp32=True)
    Jf = with_dirichlet(J, mask)
    bd = torch.from_numpy(b).cuda()
    x, n_inner, n_ref, info = solve_gmres_mixed(Jf, bd, M=M, rtol=1e-12, restart=50, maxiter=20)
    assert info == 0 and n_ref >= 2 and n_inner > 0
    ref = _direct(J, free, b)
    assert rel_err(x.cpu().numpy(), ref) < 1e-9
    x1, _, _, _ = solve_gmres_mixed(Jf, bd, M=M, rtol=1e-12, restart=50, maxiter=20, refine_max=1)
    assert rel_err(x1.cpu().numpy(), ref) > 1e-9


def test_amg_with_both_cycles_matches_fp64_cycle(c1_system):
    """A hierarchy holding both cycles applies its FP64 cycle to FP64
    vectors bit-identically to an FP64-only hierarchy."""
    import torch
    from up3d_b200.solve.linear import build_amg_preconditioner
    s = c1_system
    A = _embedded(s["A"], s["mask"])
    r = torch.from_numpy(s["b"]).cuda()
    _, Mb = build_amg_preconditioner(A, fp32="both")
    _, M64 = build_amg_preconditioner(A)
    assert torch.equal(Mb.matvec(r), M64.matvec(r))


def test_data_only_names_and_vcycle(c1_system, c1_golden):
    """up3d_picard_matrix_data / up3d_jacobian_data give the bits of
    up3d_picard_matrix / up3d_jacobian; up3d_amg_vcycle is one V-cycle
    (the AMG preconditioner's apply) and refuses a Jacobi preconditioner."""
    import ctypes
    import torch
    from up3d_b200 import _lib as L
    from up3d_b200.kernels.jacobian import PicardOperator
    from up3d_b200.solve.linear import build_amg_preconditioner, build_jacobi_preconditioner
    s = c1_system
    g = c1_golden
    op = PicardOperator(g.mesh("nodes"), g.mesh("elements"))
    rt = torch.from_numpy(g.state("mixed_m08", "rho_tilde")).cuda()
    d0 = op.assemble_matrix(rt).data
    d1 = torch.empty_like(d0)
    L.call("up3d_picard_matrix_data", op._mesh.handle, rt.data_ptr(), d1.data_ptr(), L.stream_ptr())
    assert torch.equal(d0, d1)
    args = [torch.from_numpy(g.state("mixed_m08", k)).cuda() for k in ("phi", "s_e", "s_u")]
    up = torch.from_numpy(g.state("mixed_m08", "upstream").astype(np.int64)).cuda()
    outs = []
    for name in ("up3d_jacobian", "up3d_jacobian_data"):
        d = torch.empty_like(d0)
        na, nx, nn = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        L.call(name, op._mesh.handle, args[0].data_ptr(), rt.data_ptr(), args[1].data_ptr(), args[2].data_ptr(),
               up.data_ptr(), 1.0, None, d.data_ptr(), ctypes.byref(na), ctypes.byref(nx), ctypes.byref(nn),
               L.stream_ptr())
        outs.append((d, na.value, nx.value, nn.value))
    assert torch.equal(outs[0][0], outs[1][0]) and outs[0][1:] == outs[1][1:]
    A = _embedded(s["A"], s["mask"])
    M = build_amg_preconditioner(A)[1]
    r = torch.from_numpy(s["b"]).cuda()
    z = torch.empty_like(r)
    L.call("up3d_amg_vcycle", M.handle, r.data_ptr(), z.data_ptr(), L.stream_ptr())
    assert torch.equal(z, M.matvec(r))
    Mj = build_jacobi_preconditioner(A)
    with pytest.raises(ValueError):
        L.call("up3d_amg_vcycle", Mj.handle, r.data_ptr(), z.data_ptr(), L.stream_ptr())
