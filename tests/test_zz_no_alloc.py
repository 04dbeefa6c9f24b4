"""The allocation-free CG entry point (up3d_cg_jacobi_noalloc).

It serves callers that cannot let the library call cudaMalloc/cudaFree --
a process whose device memory already belongs to another allocator or a
fixed pool, or a time-critical loop that cannot take those calls' implicit
synchronisation.  Its vectors live in one static device array that every
call reuses, so the test runs it twice in a row and checks both results
against the allocating entry point (up3d_cg + up3d_precond_jacobi) on the
same system, through the C ABI.  Collected last (file name) so that a run
stopping at the first failure has run every other test first; it also
passes alone in a fresh process.
"""

import ctypes

import numpy as np
import pytest

from conftest import has_cuda, rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]

TOL = 1e-12


@pytest.fixture(scope="module")
def system():
    """Picard matrix of a 40x10x10 bump channel, Dirichlet inflow/outflow,
    a seeded right-hand side (zero on constrained rows)."""
    import torch
    from up3d_b200 import _lib as L
    from up3d_b200.kernels.jacobian import PicardOperator
    from up3d_b200.mesh.kuhn import bump_channel
    mesh = bump_channel(40, 10, 10, amplitude=0.05, seed=0)
    op = PicardOperator(torch.from_numpy(mesh.nodes), torch.from_numpy(mesh.elements))
    A = op.assemble_matrix(torch.ones(op.n_tets, dtype=torch.float64, device="cuda"))
    mask = torch.zeros(op.n_nodes, dtype=torch.uint8, device="cuda")
    mask[torch.from_numpy(mesh.dirichlet_nodes).cuda()] = 1
    b = torch.from_numpy(np.random.default_rng(11).standard_normal(op.n_nodes)).cuda()
    b[mask.bool()] = 0.0
    csr = L.CSR(op.n_nodes, A.indptr.data_ptr(), A.indices.data_ptr(), A.data.data_ptr(),
                mask.data_ptr())
    return {"A": A, "mask": mask, "b": b, "csr": csr, "n": op.n_nodes}


def _cg_allocating(s):
    import torch
    from up3d_b200 import _lib as L
    M = ctypes.c_void_p()
    L.call("up3d_precond_jacobi", ctypes.byref(s["csr"]), ctypes.byref(M), L.stream_ptr())
    x = torch.zeros_like(s["b"])
    it, res, info = ctypes.c_int64(), ctypes.c_double(), ctypes.c_int()
    try:
        L.call("up3d_cg", ctypes.byref(s["csr"]), s["b"].data_ptr(), x.data_ptr(), 1e-12, 0.0, 5000,
               M.value, ctypes.byref(it), ctypes.byref(res), ctypes.byref(info), L.stream_ptr())
    finally:
        L.lib().up3d_precond_destroy(M.value)
    return x, int(it.value), int(info.value)


def _cg_static(s):
    import torch
    from up3d_b200 import _lib as L
    x = torch.zeros_like(s["b"])
    it, res, info = ctypes.c_int64(), ctypes.c_double(), ctypes.c_int()
    L.call("up3d_cg_jacobi_noalloc", ctypes.byref(s["csr"]), s["b"].data_ptr(), x.data_ptr(), 1e-12,
           0.0, 5000, ctypes.byref(it), ctypes.byref(res), ctypes.byref(info), L.stream_ptr())
    return x, int(it.value), int(info.value)


def test_noalloc_cg_matches_allocating_cg_twice(system):
    import torch
    x_ref, it_ref, info_ref = _cg_allocating(system)
    assert info_ref == 0
    for _ in range(2):  # the second call sees the first call's leftovers
        x, it, info = _cg_static(system)
        torch.cuda.synchronize()
        assert info == 0
        assert it == it_ref
        assert rel_err(x.cpu().numpy(), x_ref.cpu().numpy()) <= TOL


def test_noalloc_call_allocates_nothing(system):
    """After a first call on the device (which lets the driver commit the
    static array under lazy module loading), a call changes neither the
    device's free memory nor the caching allocator's total."""
    import torch
    from up3d_b200 import _lib as L
    x = torch.zeros_like(system["b"])
    it, res, info = ctypes.c_int64(), ctypes.c_double(), ctypes.c_int()

    def call():
        L.call("up3d_cg_jacobi_noalloc", ctypes.byref(system["csr"]), system["b"].data_ptr(), x.data_ptr(),
               1e-12, 0.0, 5000, ctypes.byref(it), ctypes.byref(res), ctypes.byref(info), L.stream_ptr())
    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    used0 = torch.cuda.memory_allocated()
    call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert info.value == 0
    assert free1 == free0
    assert torch.cuda.memory_allocated() == used0


def test_noalloc_rejects_oversized_systems(system):
    import torch
    from up3d_b200 import _lib as L
    big = L.CSR(L.NOALLOC_MAX_ROWS + 1, system["A"].indptr.data_ptr(), system["A"].indices.data_ptr(),
                system["A"].data.data_ptr(), None)
    x = torch.zeros_like(system["b"])
    it, res, info = ctypes.c_int64(), ctypes.c_double(), ctypes.c_int()
    with pytest.raises(ValueError, match="static limit"):
        L.call("up3d_cg_jacobi_noalloc", ctypes.byref(big), system["b"].data_ptr(), x.data_ptr(),
               1e-12, 0.0, 10, ctypes.byref(it), ctypes.byref(res), ctypes.byref(info),
               L.stream_ptr())
