"""Linear algebra on the B200 (pyfp3d/solve/linear.py): Dirichlet
elimination, the smoothed-aggregation AMG preconditioner, CG+AMG and
restarted GMRES -- SpMV, Krylov vectors and the V-cycle on the device.

Operands are ``DeviceCSR`` (optionally carrying ``dirichlet``, a uint8
mask that embeds the free-DOF system A[free][:, free] in full size, and
``extra``, the Term-3 entries outside the P1 pattern) or scipy matrices,
which are uploaded.  Vectors follow the usual rule: numpy in -> numpy out,
CUDA tensors in -> CUDA tensors out.
"""

from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from .. import _lib as L
from ..mesh.device import DeviceCSR


# ----------------------------------------------------------------- operands

def as_device_csr(A) -> DeviceCSR:
    if isinstance(A, DeviceCSR):
        return A
    import scipy.sparse as sp
    t = L.require_cuda()
    A = sp.csr_matrix(A)
    A.sort_indices()
    return DeviceCSR(L.to_device(A.indptr, t.int32), L.to_device(A.indices, t.int32),
                     L.to_device(A.data, t.float64), A.shape)


def _csr_struct(A: DeviceCSR, dirichlet=None) -> L.CSR:
    d = dirichlet if dirichlet is not None else getattr(A, "dirichlet", None)
    return L.CSR(A.shape[0], A.indptr.data_ptr(), A.indices.data_ptr(), A.data.data_ptr(),
                 None if d is None else d.data_ptr())


def with_dirichlet(A: DeviceCSR, dirichlet_mask) -> DeviceCSR:
    """The same matrix tagged with a constrained-row mask (uint8 tensor)."""
    t = L.torch()
    B = DeviceCSR(A.indptr, A.indices, A.data, A.shape)
    B.dirichlet = L.to_device(dirichlet_mask, t.uint8)
    B.extra = getattr(A, "extra", None)
    return B


def apply_dirichlet(A, b, dirichlet_nodes, dirichlet_values):
    """Principal free-DOF reduction (solve/linear.py:20-58).

    scipy input: the reference's (A_free, b_free, free, phi_dirichlet).
    DeviceCSR input: the device form (A tagged with the Dirichlet mask,
    b_free embedded in full size with zeros on constrained rows, free,
    phi_dirichlet) -- the embedded system has the same solution on the free
    DOFs without materialising the submatrix."""
    if not isinstance(A, DeviceCSR):
        import scipy.sparse as sp
        n = A.shape[0]
        is_dir = np.zeros(n, dtype=bool)
        is_dir[dirichlet_nodes] = True
        free = np.where(~is_dir)[0]
        phi_d = np.zeros(n)
        phi_d[dirichlet_nodes] = dirichlet_values
        A_csr = sp.csr_matrix(A)
        b_free = np.asarray(b)[free] - A_csr[free][:, dirichlet_nodes] @ dirichlet_values
        return A_csr[free][:, free].tocsr(), b_free, free, phi_d
    t = L.torch()
    n = A.shape[0]
    mask = t.zeros(n, dtype=t.uint8, device="cuda")
    dn = L.to_device(dirichlet_nodes, t.int64)
    mask[dn] = 1
    phi_d = t.zeros(n, dtype=t.float64, device="cuda")
    phi_d[dn] = L.to_device(dirichlet_values, t.float64)
    rhs = L.to_device(b, t.float64) - A.matvec(phi_d)
    rhs[dn] = 0.0
    free = t.nonzero(mask == 0).flatten()
    return with_dirichlet(A, mask), rhs, free, phi_d


# ----------------------------------------------------------- preconditioners

class DevicePreconditioner:
    """An up3d_precond handle; ``matvec(r)`` applies it on the device."""

    def __init__(self, handle: int, n: int, kind: str):
        self.handle = handle
        self.shape = (n, n)
        self.kind = kind

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                L.lib().up3d_precond_destroy(h)
            except Exception:
                pass
            self.handle = None

    def matvec(self, r):
        t = L.torch()
        d = L.to_device(r, t.float64)
        z = t.empty_like(d)
        L.call("up3d_precond_apply", self.handle, d.data_ptr(), z.data_ptr(), L.stream_ptr())
        return z if L.is_torch(r) else z.cpu().numpy()

    __call__ = matvec

    def refresh(self, A, dirichlet=None):
        """New values for an AMG hierarchy from a matrix with the pattern
        and Dirichlet mask of its setup matrix (up3d_amg_refresh): equal,
        bit for bit, to a fresh build_amg_preconditioner on A.  ValueError
        when the pattern or mask differ."""
        if not self.kind.startswith("amg"):
            raise TypeError("refresh applies to AMG preconditioners")
        Ad = as_device_csr(A)
        L.call("up3d_amg_refresh", self.handle, ctypes.byref(_csr_struct(Ad, dirichlet)), L.stream_ptr())
        return self


class AMGHierarchy:
    """The ``ml`` object of build_amg_preconditioner: level sizes and
    complexity of the device hierarchy."""

    def __init__(self, M: DevicePreconditioner):
        info = L.AmgInfo()
        L.call("up3d_amg_get_info", M.handle, ctypes.byref(info))
        self.n_levels = int(info.n_levels)
        self.level_rows = [int(info.level_rows[i]) for i in range(min(self.n_levels, 16))]
        self.operator_complexity = float(info.operator_complexity)
        self.n_coarse = int(info.n_coarse)
        self._M = M

    def aspreconditioner(self):
        return self._M

    def __repr__(self):
        return (f"AMGHierarchy(levels={self.n_levels}, rows={self.level_rows}, "
                f"operator_complexity={self.operator_complexity:.3f})")


_AMG_KINDS = {False: ("amg", 0), True: ("amg32", 1), "both": ("amg64+32", 2)}


def build_amg_preconditioner(A, fp32=False, max_coarse: int = 500, max_levels: int = 10,
                             presmooth: int = 2, postsmooth: int = 2, dirichlet=None):
    """Smoothed-aggregation AMG (solve/linear.py:61-81); returns (ml, M).
    fp32: False (FP64 cycle), True (FP32 cycle, FP64 coarsest solve) or
    "both" (FP64 vectors take the FP64 cycle, FP32 vectors the FP32 one).
    Setup is deterministic (no random start vector), so repeated setups on
    a bit-identical matrix give bit-identical hierarchies."""
    Ad = as_device_csr(A)
    kind, code = _AMG_KINDS[fp32]
    opts = L.AmgOptions(int(max_levels), int(max_coarse), int(presmooth), int(postsmooth), code)
    h = ctypes.c_void_p()
    L.call("up3d_amg_setup", ctypes.byref(_csr_struct(Ad, dirichlet)), ctypes.byref(opts),
           ctypes.byref(h), L.stream_ptr())
    M = DevicePreconditioner(h.value, Ad.shape[0], kind)
    return AMGHierarchy(M), M


def amg_for(A, M: Optional[DevicePreconditioner] = None, fp32=False, dirichlet=None):
    """The AMG preconditioner of A: M refreshed with A's values when M was
    set up (with the same precision) on A's pattern, else a new setup.
    Returns the preconditioner."""
    kind = _AMG_KINDS[fp32][0]
    if M is not None and M.kind == kind:
        try:
            return M.refresh(A, dirichlet)
        except ValueError:
            pass
    return build_amg_preconditioner(A, fp32=fp32, dirichlet=dirichlet)[1]


def build_jacobi_preconditioner(A, dirichlet=None) -> DevicePreconditioner:
    Ad = as_device_csr(A)
    h = ctypes.c_void_p()
    L.call("up3d_precond_jacobi", ctypes.byref(_csr_struct(Ad, dirichlet)), ctypes.byref(h),
           L.stream_ptr())
    return DevicePreconditioner(h.value, Ad.shape[0], "jacobi")


def build_ilu_preconditioner(A, drop_tol: float = 1e-4, fill_factor: float = 10.0, dirichlet=None,
                             sweeps: int = 5, tri_sweeps: int = 3) -> DevicePreconditioner:
    """Incomplete-LU preconditioner (solve/linear.py:84-131) on the device:
    ILU(0) on A's own pattern by fixed-point sweeps, applied with Jacobi
    sweeps on each triangle (up3d_precond_ilu0).  The reference's threshold
    ILU (scipy spilu with drop_tol and fill_factor, a serial host
    factorisation) has no device form; drop_tol and fill_factor are
    accepted and not used: ILU(0) keeps no fill and drops nothing.  A
    non-finite factorisation is redone shifted by 1e-3 mean|a_ii| (the
    reference's last fallback).  Returns a DevicePreconditioner (FP64)."""
    Ad = as_device_csr(A)
    h = ctypes.c_void_p()
    L.call("up3d_precond_ilu0", ctypes.byref(_csr_struct(Ad, dirichlet)), int(sweeps), int(tri_sweeps),
           ctypes.byref(h), L.stream_ptr())
    return DevicePreconditioner(h.value, Ad.shape[0], "ilu0")


def ilu_factors(M: DevicePreconditioner, nnz: int):
    """(values on A's pattern, diagonal shift) of an ILU(0) preconditioner."""
    t = L.torch()
    lu = t.empty(nnz, dtype=t.float64, device="cuda")
    shift = ctypes.c_double()
    L.call("up3d_precond_ilu0_factors", M.handle, lu.data_ptr(), ctypes.byref(shift), L.stream_ptr())
    return lu, float(shift.value)


# ------------------------------------------------------------------ solvers

def _extra_struct(A: DeviceCSR):
    X = getattr(A, "extra", None)
    if X is None:
        return None
    return ctypes.byref(L.CSR(X.shape[0], X.indptr.data_ptr(), X.indices.data_ptr(),
                              X.data.data_ptr(), None))


def solve_gmres(A, b, M=None, rtol: float = 1e-6, atol: float = 0.0, x0=None, restart: int = 60,
                maxiter: int = 50, on_fail: str = "retry") -> Tuple[object, int, int]:
    """Restarted preconditioned GMRES (solve/linear.py:134-201): returns
    (x, n_inner_iterations, info); on_fail="retry" retries once at doubled
    restart and then raises RuntimeError, "return" hands back the iterate."""
    t = L.require_cuda()
    Ad = as_device_csr(A)
    host = not L.is_torch(b)
    d_b = L.to_device(b, t.float64)
    x = t.zeros_like(d_b) if x0 is None else L.to_device(x0, t.float64).clone()
    if M is not None and not isinstance(M, DevicePreconditioner):
        raise TypeError("M must be a DevicePreconditioner (build_amg_preconditioner / "
                        "build_jacobi_preconditioner)")

    def run(rs):
        inner, resid, info = ctypes.c_int64(), ctypes.c_double(), ctypes.c_int()
        L.call("up3d_gmres", ctypes.byref(_csr_struct(Ad)), _extra_struct(Ad), d_b.data_ptr(),
               x.data_ptr(), float(rtol), float(atol), int(rs), int(maxiter),
               None if M is None else M.handle, ctypes.byref(inner), ctypes.byref(resid),
               ctypes.byref(info), L.stream_ptr())
        return int(inner.value), int(info.value)

    n_it, info = run(restart)
    if info != 0 and on_fail == "retry":
        n2, info = run(2 * restart)
        if info != 0:
            raise RuntimeError(f"GMRES did not converge (info={info}) after {n_it} + {n2} inner "
                               f"iterations (restart {restart} then {2 * restart}, rtol={rtol:g})")
        n_it += n2
    return (x.cpu().numpy() if host else x), n_it, info


def solve_gmres_mixed(A, b, M=None, rtol: float = 1e-6, atol: float = 0.0, x0=None, restart: int = 50,
                      maxiter: int = 20, refine_max: int = 10, inner_rtol: float = 1e-4,
                      values32=None) -> Tuple[object, int, int, int]:
    """Mixed-precision GMRES with FP64 iterative refinement (up3d_gmres_ir):
    inner GMRES(restart) in FP32 on A's FP32 values with M applied in FP32,
    outer residual, update and convergence test in FP64.  ``values32`` =
    (data32, extra32) reuses FP32 copies of A's values.  Returns (x,
    n_inner_iterations, n_refinements, info)."""
    t = L.require_cuda()
    Ad = as_device_csr(A)
    host = not L.is_torch(b)
    d_b = L.to_device(b, t.float64)
    x = t.zeros_like(d_b) if x0 is None else L.to_device(x0, t.float64).clone()
    if M is not None and not isinstance(M, DevicePreconditioner):
        raise TypeError("M must be a DevicePreconditioner")
    X = getattr(Ad, "extra", None)
    if values32 is None:
        values32 = (Ad.data.to(t.float32), None if X is None else X.data.to(t.float32))
    d32, x32 = values32
    inner, outer, resid, info = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double(), ctypes.c_int()
    L.call("up3d_gmres_ir", ctypes.byref(_csr_struct(Ad)), _extra_struct(Ad), d32.data_ptr(),
           None if x32 is None else x32.data_ptr(), d_b.data_ptr(), x.data_ptr(), float(rtol),
           float(atol), int(restart), int(maxiter), int(refine_max), float(inner_rtol),
           None if M is None else M.handle, ctypes.byref(inner), ctypes.byref(outer),
           ctypes.byref(resid), ctypes.byref(info), L.stream_ptr())
    return (x.cpu().numpy() if host else x), int(inner.value), int(outer.value), int(info.value)


def solve_cg(A, b, M=None, rtol: float = 1e-10, atol: float = 0.0, maxiter: int = 500, x0=None):
    """Preconditioned CG; returns (x, n_iter, info)."""
    t = L.require_cuda()
    Ad = as_device_csr(A)
    host = not L.is_torch(b)
    d_b = L.to_device(b, t.float64)
    x = t.zeros_like(d_b) if x0 is None else L.to_device(x0, t.float64).clone()
    it, resid, info = ctypes.c_int64(), ctypes.c_double(), ctypes.c_int()
    L.call("up3d_cg", ctypes.byref(_csr_struct(Ad)), d_b.data_ptr(), x.data_ptr(), float(rtol),
           float(atol), int(maxiter), None if M is None else M.handle, ctypes.byref(it),
           ctypes.byref(resid), ctypes.byref(info), L.stream_ptr())
    return (x.cpu().numpy() if host else x), int(it.value), int(info.value)


def solve_cg_amg(A, b, rtol: float = 1e-10, maxiter: int = 500):
    """CG + smoothed-aggregation AMG (solve/linear.py:204-239): returns
    (x, n_iterations); RuntimeError if CG does not converge."""
    _, M = build_amg_preconditioner(A)
    x, n_it, info = solve_cg(A, b, M=M, rtol=rtol, maxiter=maxiter)
    if info != 0:
        raise RuntimeError(f"CG did not converge (info={info}) after {n_it} iterations")
    return x, n_it
