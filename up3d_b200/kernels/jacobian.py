"""PicardOperator on the B200: the per-mesh workspace of the Picard matrix,
residual and exact Newton Jacobian, with the reference's signatures
(pyfp3d/kernels/jacobian.py:231-375).

Arrays in, same kind out: numpy arguments give numpy arrays and
``scipy.sparse.csr_matrix`` results (host copies, as the reference returns);
CUDA-tensor arguments give CUDA tensors and ``DeviceCSR`` results with no
host round trip.  Returned vectors are views into workspace buffers that the
next call of the same method overwrites, as in the reference.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from .. import _lib as L
from ..mesh.device import DeviceCSR, get_mesh


class PicardOperator:
    """B200 PicardOperator (kernels/jacobian.py:231-375).

    Usage (Picard outer loop):
        op = PicardOperator(nodes, elements)
        grad, q2 = op.velocities(phi)
        rho = density_field(q2 / u_inf**2, m_inf)
        A = op.assemble_matrix(rho)
        R = op.assemble_residual(phi, rho)
    """

    def __init__(self, nodes, elements, *, mesh=None):
        """`mesh` (keyword only, not in the reference's signature): a
        DeviceMesh of these nodes and elements to work on instead of the
        shared handle looked up from the arrays."""
        t = L.require_cuda()
        self._mesh = mesh if mesh is not None else get_mesh(nodes, elements)
        m = self._mesh
        self.n_nodes = m.n_nodes
        self.n_tets = m.n_tets
        self.elements = m.elements
        self._host = not L.is_torch(nodes)
        E, N = self.n_tets, self.n_nodes
        self._grad_d = t.empty((E, 3), dtype=t.float64, device="cuda")
        self._q2_d = t.empty(E, dtype=t.float64, device="cuda")
        self._R_d = t.empty(N, dtype=t.float64, device="cuda")
        self._grad = np.empty((E, 3))
        self._q2 = np.empty(E)
        self._R = np.empty(N)
        self.rho_ones = np.ones(E)
        self._B = self._V = None
        self._e2c = None
        self._pattern_cache = None
        self.newton_nnz = None
        self.n_term3_active = None
        self.n_term3_extra = None

    # ---------------------------------------------------------- attributes

    @property
    def mesh(self):
        return self._mesh

    @property
    def B(self):
        if self._B is None:
            B, V = self._mesh.geometry()
            self._B, self._V = (B.cpu().numpy(), V.cpu().numpy()) if self._host else (B, V)
        return self._B

    @property
    def V(self):
        self.B
        return self._V

    @property
    def color_offsets(self):
        return self._mesh.coloring()[0]

    @property
    def color_elems(self):
        return self._mesh.coloring()[1]

    @property
    def n_colors(self):
        return self._mesh.coloring()[2]

    @property
    def elem_to_csr(self):
        if self._e2c is None:
            d = self._mesh.elem_to_csr()
            self._e2c = d.cpu().numpy() if self._host else d
        return self._e2c

    @property
    def _pattern(self):
        if self._pattern_cache is None:
            import scipy.sparse as sp
            m = self._mesh
            self._pattern_cache = sp.csr_matrix(
                (np.zeros(m.nnz), m.indices.cpu().numpy(), m.indptr.cpu().numpy()),
                shape=(self.n_nodes, self.n_nodes))
        return self._pattern_cache

    # ---------------------------------------------------------- helpers

    def _dev(self, x, dtype=None):
        t = L.torch()
        return None if x is None else L.to_device(x, dtype or t.float64)

    def _host_out(self, *pairs):
        out = []
        for dev, host in pairs:
            host[...] = dev.cpu().numpy()
            out.append(host)
        return tuple(out)

    def _csr_result(self, indptr, indices, data, host):
        if host:
            import scipy.sparse as sp
            return sp.csr_matrix((data.cpu().numpy(), indices.cpu().numpy(), indptr.cpu().numpy()),
                                 shape=(self.n_nodes, self.n_nodes))
        return DeviceCSR(indptr, indices, data, (self.n_nodes, self.n_nodes))

    # ---------------------------------------------------------- methods

    def velocities(self, phi):
        """Element-constant grad(phi)_e and q^2_e (kernels/jacobian.py:264-270)."""
        d_phi = self._dev(phi)
        L.call("up3d_velocities", self._mesh.handle, d_phi.data_ptr(), self._grad_d.data_ptr(),
               self._q2_d.data_ptr(), L.stream_ptr())
        if L.is_torch(phi):
            return self._grad_d, self._q2_d
        return self._host_out((self._grad_d, self._grad), (self._q2_d, self._q2))

    def assemble_matrix(self, rho_tilde: Optional[object] = None):
        """Weighted stiffness matrix (kernels/jacobian.py:272-286); None means
        rho == 1."""
        t = L.torch()
        host = self._host if rho_tilde is None else not L.is_torch(rho_tilde)
        d_rt = self._dev(rho_tilde)
        data = t.empty(self._mesh.nnz, dtype=t.float64, device="cuda")
        L.call("up3d_picard_matrix", self._mesh.handle, L.ptr(d_rt), data.data_ptr(), L.stream_ptr())
        return self._csr_result(self._mesh.indptr, self._mesh.indices, data, host)

    def assemble_newton_jacobian(self, phi, rho_tilde, s_e, s_u, upstream, u_inf: float = 1.0,
                                 lim_mask=None):
        """Exact Newton Jacobian dR/dphi (kernels/jacobian.py:288-359): Terms
        1+2 on the P1 pattern plus the active-set Term 3; records
        newton_nnz and n_term3_active.  Inputs are not modified."""
        t = L.torch()
        host = not L.is_torch(phi)
        d_phi, d_rt = self._dev(phi), self._dev(rho_tilde)
        d_se, d_su = self._dev(s_e), self._dev(s_u)
        d_up = L.to_device(upstream, t.int64)
        d_lim = None if lim_mask is None else L.to_device(lim_mask, t.uint8)
        data = t.empty(self._mesh.nnz, dtype=t.float64, device="cuda")
        na, nx, nnz = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        L.call("up3d_jacobian", self._mesh.handle, d_phi.data_ptr(), d_rt.data_ptr(), d_se.data_ptr(),
               d_su.data_ptr(), d_up.data_ptr(), float(u_inf), L.ptr(d_lim), data.data_ptr(),
               ctypes.byref(na), ctypes.byref(nx), ctypes.byref(nnz), L.stream_ptr())
        self.n_term3_active = int(na.value)
        self.n_term3_extra = int(nx.value)
        self.newton_nnz = int(nnz.value)
        if self.n_term3_active == 0:
            return self._csr_result(self._mesh.indptr, self._mesh.indices, data, host)
        indptr = t.empty(self.n_nodes + 1, dtype=t.int32, device="cuda")
        indices = t.empty(self.newton_nnz, dtype=t.int32, device="cuda")
        merged = t.empty(self.newton_nnz, dtype=t.float64, device="cuda")
        L.call("up3d_jacobian_export", self._mesh.handle, data.data_ptr(), indptr.data_ptr(),
               indices.data_ptr(), merged.data_ptr(), L.stream_ptr())
        return self._csr_result(indptr, indices, merged, host)

    def assemble_residual(self, phi, rho_tilde=None):
        """Nonlinear residual (kernels/jacobian.py:361-375); also refreshes
        the velocity workspace like the reference."""
        d_phi, d_rt = self._dev(phi), self._dev(rho_tilde)
        L.call("up3d_residual", self._mesh.handle, d_phi.data_ptr(), L.ptr(d_rt), self._R_d.data_ptr(),
               self._grad_d.data_ptr(), self._q2_d.data_ptr(), L.stream_ptr())
        if L.is_torch(phi):
            return self._R_d
        self._host_out((self._grad_d, self._grad), (self._q2_d, self._q2))
        return self._host_out((self._R_d, self._R))[0]
