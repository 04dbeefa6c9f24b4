"""Device ILU(0) preconditioner (build_ilu_preconditioner, up3d_precond_ilu0,
in place of the reference's host threshold ILU, solve/linear.py:84-131):
the fixed-point factors reach the sequential ILU(0) factors on the P1
pattern (with the Dirichlet embedding), GMRES with it reaches the direct
solution, a zero pivot falls back to the diagonal shift, and a pattern
without a diagonal is refused."""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from conftest import has_cuda, rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]


def _ilu0_host(A):
    """Sequential ILU(0) (IKJ order) on A's pattern: one array of L
    (strictly lower, unit diagonal implied) and U (upper) values."""
    A = sp.csr_matrix(A)
    A.sort_indices()
    ip, ix = A.indptr, A.indices
    lu = A.data.astype(np.float64).copy()
    pos = [dict(zip(ix[ip[r]:ip[r + 1]], range(ip[r], ip[r + 1]))) for r in range(A.shape[0])]
    for i in range(A.shape[0]):
        for q in range(ip[i], ip[i + 1]):
            k = ix[q]
            if k >= i:
                break
            lu[q] /= lu[pos[k][k]]
            for q2 in range(q + 1, ip[i + 1]):
                j = ix[q2]
                if j in pos[k]:
                    lu[q2] -= lu[q] * lu[pos[k][j]]
    return lu


def _system():
    import torch
    from up3d_b200.kernels.jacobian import PicardOperator
    from up3d_b200.mesh.kuhn import bump_channel, seeded_state
    from up3d_b200.physics.isentropic import density_field
    m = bump_channel(10, 4, 3, amplitude=0.08, seed=1)
    op = PicardOperator(torch.from_numpy(m.nodes).cuda(), torch.from_numpy(m.elements).cuda())
    _, q2 = op.velocities(torch.from_numpy(seeded_state(m, 1)).cuda())
    A = op.assemble_matrix(density_field(q2, 0.6))
    mask = torch.zeros(m.n_nodes, dtype=torch.uint8, device="cuda")
    mask[torch.from_numpy(m.dirichlet_nodes).cuda()] = 1
    return m, A, mask


def _embedded(A, mask):
    S = A.to_scipy().tolil()
    d = np.flatnonzero(mask.cpu().numpy())
    for r in d:
        S.rows[r] = [r]
        S.data[r] = [1.0]
    S = S.tocsr()
    keep = np.ones(S.shape[0], dtype=bool)
    keep[d] = False
    S = sp.csr_matrix(S.multiply(keep[None, :])) + sp.diags((~keep).astype(float))
    return S


def test_fixed_point_factors_reach_sequential_ilu0():
    from up3d_b200.solve.linear import build_ilu_preconditioner, ilu_factors, with_dirichlet
    m, A, mask = _system()
    M = build_ilu_preconditioner(with_dirichlet(A, mask), sweeps=40)
    lu, shift = ilu_factors(M, A.nnz)
    assert shift == 0.0
    # the embedded operator on A's pattern (zeros kept where the mask drops)
    S = A.to_scipy()
    E = _embedded(A, mask)
    rows = np.repeat(np.arange(S.shape[0]), np.diff(S.indptr))
    Ep = sp.csr_matrix((np.asarray(E[rows, S.indices]).ravel(), S.indices, S.indptr), shape=S.shape)
    ref = _ilu0_host(Ep)
    assert rel_err(lu.cpu().numpy(), ref) < 1e-12
    # fewer sweeps: an approximation, still finite
    M5 = build_ilu_preconditioner(with_dirichlet(A, mask))
    lu5, _ = ilu_factors(M5, A.nnz)
    assert np.isfinite(lu5.cpu().numpy()).all()


def test_gmres_with_ilu_reaches_the_direct_solution():
    import torch
    from up3d_b200.solve.linear import build_ilu_preconditioner, solve_gmres, with_dirichlet
    m, A, mask = _system()
    Af = with_dirichlet(A, mask)
    b = np.random.default_rng(3).standard_normal(m.n_nodes)
    b[m.dirichlet_nodes] = 0.0
    M = build_ilu_preconditioner(Af)
    x, n_it, info = solve_gmres(Af, torch.from_numpy(b).cuda(), M=M, rtol=1e-12, restart=60, maxiter=20)
    assert info == 0
    ref = spla.spsolve(_embedded(A, mask).tocsc(), b)
    assert rel_err(x.cpu().numpy(), ref) < 1e-9
    _, n_plain, _ = solve_gmres(Af, torch.from_numpy(b).cuda(), M=None, rtol=1e-12, restart=60, maxiter=20)
    assert n_it < n_plain
    with pytest.raises(NotImplementedError):
        from up3d_b200.solve.linear import solve_gmres_mixed
        solve_gmres_mixed(Af, torch.from_numpy(b).cuda(), M=M, rtol=1e-8)


def test_zero_pivot_takes_the_diagonal_shift_and_missing_diagonal_is_refused():
    import torch
    from up3d_b200.mesh.device import DeviceCSR
    from up3d_b200.solve.linear import build_ilu_preconditioner, ilu_factors
    m, A, mask = _system()
    S = A.to_scipy()
    S.sort_indices()
    data = S.data.copy()
    r0 = 7
    d0 = S.indptr[r0] + int(np.flatnonzero(S.indices[S.indptr[r0]:S.indptr[r0 + 1]] == r0)[0])
    data[d0] = 0.0
    Z = DeviceCSR(torch.from_numpy(S.indptr.astype(np.int32)).cuda(), torch.from_numpy(S.indices.astype(np.int32)).cuda(),
                  torch.from_numpy(data).cuda(), S.shape)
    M = build_ilu_preconditioner(Z)
    lu, shift = ilu_factors(M, S.nnz)
    assert shift > 0.0 and np.isfinite(lu.cpu().numpy()).all()
    # a row without its diagonal
    T = sp.csr_matrix(S.copy())
    T = T.tolil()
    T[r0, r0] = 0.0
    T = sp.csr_matrix(T)
    T.eliminate_zeros()
    Y = DeviceCSR(torch.from_numpy(T.indptr.astype(np.int32)).cuda(), torch.from_numpy(T.indices.astype(np.int32)).cuda(),
                  torch.from_numpy(T.data.astype(np.float64)).cuda(), T.shape)
    with pytest.raises(ValueError, match="diagonal"):
        build_ilu_preconditioner(Y)
    with pytest.raises(ValueError):
        build_ilu_preconditioner(Z, sweeps=0)
