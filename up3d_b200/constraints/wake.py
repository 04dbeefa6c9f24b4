"""Wake master-slave elimination and Kutta targets on the B200, with the
reference's signatures (pyfp3d/constraints/wake.py:32-212).

The cut mesh appends the "+"-side copies of the wake-sheet nodes after the
original nodes, so the reduced unknowns are the original nodes:
phi_cut = T phi_red + g(Gamma).  ``WakeConstraint`` forms A_red = T^T A T and
the Gamma columns H = T^T A G on the device (``up3d_wake_*``): a host
symbolic phase per A pattern (kept while the pattern repeats) and a device
gather per call.  Arrays in, same kind out: scipy / numpy inputs give scipy
/ numpy results (host copies, as the reference returns), ``DeviceCSR`` /
CUDA tensors give device results.
"""

from __future__ import annotations

import ctypes
import zlib

import numpy as np

from .. import _lib as L
from ..mesh.device import DeviceCSR, device_view


class _Plan:
    """One up3d_wake handle: the fold map and the reduction plans of one A
    pattern."""

    def __init__(self, wc, n_cut, indptr, indices, device):
        h = ctypes.c_void_p()
        m = np.ascontiguousarray(wc.master_nodes, dtype=np.int64)
        s = np.ascontiguousarray(wc.slave_nodes, dtype=np.int64)
        st = np.ascontiguousarray(wc.node_station, dtype=np.int64)
        ip = np.ascontiguousarray(indptr, dtype=np.int64)
        ix = np.ascontiguousarray(indices, dtype=np.int32)
        L.call("up3d_wake_create", n_cut, int(wc.n_nodes_orig), len(s), m.ctypes.data, s.ctypes.data,
               st.ctypes.data, int(wc.n_stations), ip.ctypes.data, ix.ctypes.data, device, ctypes.byref(h))
        self.handle = h.value
        n_red, nnz_red, nnz_h, n_st = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
        L.call("up3d_wake_info", self.handle, ctypes.byref(n_red), ctypes.byref(nnz_red), ctypes.byref(nnz_h),
               ctypes.byref(n_st))
        self.n_red, self.nnz_red, self.nnz_h, self.n_st = n_red.value, nnz_red.value, nnz_h.value, n_st.value
        self.nnz_a = int(ip[-1])
        p = [ctypes.c_void_p() for _ in range(4)]
        L.call("up3d_wake_patterns", self.handle, *[ctypes.byref(x) for x in p])
        self.red_indptr = device_view(p[0].value, (self.n_red + 1,), np.int32).clone()
        self.red_indices = device_view(p[1].value, (self.nnz_red,), np.int32).clone() if self.nnz_red else \
            L.torch().empty(0, dtype=L.torch().int32, device="cuda")
        self.h_indptr = device_view(p[2].value, (self.n_red + 1,), np.int32).clone()
        self.h_indices = device_view(p[3].value, (self.nnz_h,), np.int32).clone() if self.nnz_h else \
            L.torch().empty(0, dtype=L.torch().int32, device="cuda")

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                L.lib().up3d_wake_destroy(h)
            except Exception:
                pass
            self.handle = None


def _pattern_key(indptr, indices):
    if L.is_torch(indices):
        t = L.torch()
        return ("dev", int(indices.numel()), int(indptr.data_ptr()), int(indices.data_ptr()),
                int(indices.to(t.int64).sum()), int(indptr[-1]))
    ix = np.ascontiguousarray(indices, dtype=np.int32)
    ip = np.ascontiguousarray(indptr, dtype=np.int64)
    return ("host", len(ix), zlib.crc32(ip.tobytes()), zlib.crc32(ix.tobytes()))


class WakeConstraint:
    """Precomputed elimination operator for one cut mesh
    (constraints/wake.py:32-127)."""

    def __init__(self, A, wc):
        t = L.require_cuda()
        n_cut = A.shape[0]
        n_red = int(wc.n_nodes_orig)
        n_slaves = len(wc.slave_nodes)
        if n_cut != n_red + n_slaves:
            raise ValueError(f"A is {n_cut}x{n_cut} but WakeCut implies {n_red} + {n_slaves} nodes")
        self.wc = wc
        self.n_reduced = n_red
        self._n_cut = n_cut
        self._device = t.cuda.current_device()
        self._plans = {}
        self._T = None
        self.update_matrix(A)

    @property
    def T(self):
        """T (n_cut x n_red) as scipy CSR: identity on the original nodes,
        T[slave_k, master_k] = 1."""
        if self._T is None:
            import scipy.sparse as sp
            wc = self.wc
            rows = np.concatenate([np.arange(self.n_reduced, dtype=np.int64), wc.slave_nodes])
            cols = np.concatenate([np.arange(self.n_reduced, dtype=np.int64), wc.master_nodes])
            self._T = sp.coo_matrix((np.ones(self._n_cut), (rows, cols)),
                                    shape=(self._n_cut, self.n_reduced)).tocsr()
        return self._T

    def _plan_for(self, indptr, indices):
        key = _pattern_key(indptr, indices)
        plan = self._plans.get(key)
        if plan is None:
            ip = indptr.cpu().numpy() if L.is_torch(indptr) else indptr
            ix = indices.cpu().numpy() if L.is_torch(indices) else indices
            if len(self._plans) >= 4:
                self._plans.pop(next(iter(self._plans)))
            plan = self._plans[key] = _Plan(self.wc, self._n_cut, ip, ix, self._device)
        return plan

    def _reduce(self, A):
        """(plan, red_data, h_data, host) on the device."""
        t = L.torch()
        host = not isinstance(A, DeviceCSR)
        if host:
            import scipy.sparse as sp
            A = sp.csr_matrix(A)
            indptr, indices = A.indptr, A.indices
            data = t.from_numpy(np.ascontiguousarray(A.data, dtype=np.float64)).cuda()
        else:
            indptr, indices, data = A.indptr, A.indices, A.data
        plan = self._plan_for(indptr, indices)
        if plan.nnz_a != int(data.numel()):
            raise ValueError("A's values do not match its pattern")
        red = t.empty(plan.nnz_red, dtype=t.float64, device="cuda")
        h = t.empty(plan.nnz_h, dtype=t.float64, device="cuda")
        L.call("up3d_wake_reduce", plan.handle, data.data_ptr(), red.data_ptr() if plan.nnz_red else None,
               h.data_ptr() if plan.nnz_h else None, L.stream_ptr())
        return plan, red, h, host

    def reduce_operator(self, A):
        """(T^T A T, T^T A G) (constraints/wake.py:59-82)."""
        plan, red, h, host = self._reduce(A)
        n_red, n_st = self.n_reduced, self.wc.n_stations
        A_red = DeviceCSR(plan.red_indptr, plan.red_indices, red, (n_red, n_red))
        H = DeviceCSR(plan.h_indptr, plan.h_indices, h, (n_red, n_st))
        if host:
            return A_red.to_scipy(), H.to_scipy()
        return A_red, H

    def update_matrix(self, A) -> None:
        """A_reduced and the per-station right-hand-side vectors h_j for a
        new A on the same cut mesh (constraints/wake.py:84-97)."""
        plan, red, h, host = self._reduce(A)
        n_red, n_st = self.n_reduced, self.wc.n_stations
        self._plan, self._h_data = plan, h
        A_red = DeviceCSR(plan.red_indptr, plan.red_indices, red, (n_red, n_red))
        H = DeviceCSR(plan.h_indptr, plan.h_indices, h, (n_red, n_st))
        self.A_reduced = A_red.to_scipy() if host else A_red
        self._h = H.to_scipy().T.toarray() if host else None
        self._host = host

    def reduced_rhs(self, b, gamma):
        """T^T b - sum_j Gamma_j h_j (constraints/wake.py:99-102)."""
        t = L.torch()
        d_b = L.to_device(b, t.float64)
        g = np.atleast_1d(np.asarray(gamma.cpu() if L.is_torch(gamma) else gamma, dtype=np.float64))
        d_g = t.from_numpy(np.ascontiguousarray(g)).cuda()
        out = t.empty(self.n_reduced, dtype=t.float64, device="cuda")
        plan = self._plan
        L.call("up3d_wake_reduced_rhs", plan.handle, d_b.data_ptr(), d_g.data_ptr(),
               self._h_data.data_ptr() if plan.nnz_h else None, out.data_ptr(), L.stream_ptr())
        return out if L.is_torch(b) else out.cpu().numpy()

    def expand(self, phi_red, gamma):
        """phi on the cut mesh (constraints/wake.py:104-112)."""
        t = L.torch()
        d_p = L.to_device(phi_red, t.float64)
        g = np.atleast_1d(np.asarray(gamma.cpu() if L.is_torch(gamma) else gamma, dtype=np.float64))
        d_g = t.from_numpy(np.ascontiguousarray(g)).cuda()
        out = t.empty(self._n_cut, dtype=t.float64, device="cuda")
        L.call("up3d_wake_expand", self._plan.handle, d_p.data_ptr(), d_g.data_ptr(), out.data_ptr(),
               L.stream_ptr())
        return out if L.is_torch(phi_red) else out.cpu().numpy()

    def to_reduced_dirichlet(self, dirichlet_nodes, dirichlet_values):
        """Cut-mesh Dirichlet data on the reduced space: slave entries
        dropped (constraints/wake.py:114-127)."""
        nodes = np.asarray(dirichlet_nodes, dtype=np.int64)
        keep = nodes < self.n_reduced
        red_nodes, idx = np.unique(nodes[keep], return_index=True)
        return red_nodes, np.asarray(dirichlet_values, dtype=np.float64)[keep][idx]


def kutta_targets(phi, wc):
    """Per-station mean of phi[upper probe] - phi[lower probe]
    (constraints/wake.py:196-212)."""
    if L.is_torch(phi):
        t = L.torch()
        up = t.as_tensor(wc.kutta_upper, device=phi.device)
        lo = t.as_tensor(wc.kutta_lower, device=phi.device)
        st = t.as_tensor(wc.te_station, device=phi.device)
        jumps = phi[up] - phi[lo]
        sums = t.zeros(wc.n_stations, dtype=phi.dtype, device=phi.device).index_add(0, st, jumps)
        counts = t.bincount(st, minlength=wc.n_stations).to(phi.dtype)
        return sums / counts
    jumps = np.asarray(phi)[wc.kutta_upper] - np.asarray(phi)[wc.kutta_lower]
    sums = np.bincount(wc.te_station, weights=jumps, minlength=wc.n_stations)
    return sums / np.bincount(wc.te_station, minlength=wc.n_stations)
