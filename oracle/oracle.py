"""CPU ORACLE of the pyfp3d element-loop hot path (test infrastructure).

Python face of ``up3d_oracle.c``: the reference's operator objects
(``PicardOperator``, ``UpwindOperator``, the isentropic field functions)
restated over the C kernels, plus ``chain`` -- the residual + Jacobian
composition of ``NewtonWorkspace.eval_residual`` / ``assemble_coupled``
(``pyfp3d/solve/newton.py:345-372``, ``:430-452``) without a wake.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU baseline use
this module; the CUDA product never imports it.  The glue follows the
reference's own host code: numpy for per-array arithmetic and scipy's
COO -> CSR summation for the Term-3 merge (``kernels/jacobian.py:344-358``).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

GAMMA = 1.4

_lib = None


def build() -> Path:
    """Compile liboracle.so (needs gcc with OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


_d = ctypes.c_double
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_p = ctypes.c_void_p


def _declare(L):
    sig = {
        "orc_q2_at_mach": (_d, [_d, _d, _d]),
        "orc_density_field": (None, [_p, _i64, _d, _d, _p]),
        "orc_mach2_field": (None, [_p, _i64, _d, _d, _p]),
        "orc_limit_q2_field": (None, [_p, _i64, _d, _d, _d, _p]),
        "orc_drho_field": (None, [_p, _i64, _d, _d, _p]),
        "orc_element_geometry": (_i64, [_p, _p, _i64, _p, _p]),
        "orc_face_adjacency": (None, [_p, _i64, _p]),
        "orc_centroids": (None, [_p, _p, _i64, _p]),
        "orc_node_to_element": (None, [_p, _i64, _i64, _p, _p]),
        "orc_greedy_coloring": (_i32, [_p, _i64, _i64, _p]),
        "orc_color_partition": (None, [_p, _i64, _i32, _p, _p]),
        "orc_csr_pattern": (_i64, [_p, _i64, _i64, _p, _p]),
        "orc_elem_to_csr": (None, [_p, _i64, _p, _p, _p]),
        "orc_velocities": (None, [_p, _p, _p, _i64, _p, _p]),
        "orc_upstream": (None, [_p, _p, _p, _p, _p, _i64, ctypes.c_int, _p]),
        "orc_rho_tilde": (None, [_p, _p, _p, _i64, _d, _d, _d, _d, _d, _p, _p]),
        "orc_classify": (None, [_p, _p, _p, _i64, _d, _d, _d, _d, _d, _p]),
        "orc_rho_tilde_frozen": (None, [_p, _p, _p, _p, _i64, _d, _d, _d, _d, _d, _p, _p]),
        "orc_sens_frozen": (None, [_p, _p, _p, _p, _i64, _d, _d, _d, _d, _d, _p, _p]),
        "orc_sens": (None, [_p, _p, _p, _i64, _d, _d, _d, _d, _d, _p, _p]),
        "orc_residual": (None, [_p, _p, _i32, _p, _p, _p, _p, _p, _i64, _p]),
        "orc_matrix_data": (None, [_p, _p, _i32, _p, _p, _p, _p, _i64, _p]),
        "orc_jacobian_data": (None, [_p, _p, _i32, _p, _p, _p, _p, _p, _p, _d, _i64, _p]),
        "orc_term3_coo": (None, [_p, _i64, _p, _p, _p, _p, _p, _p, _d, _p, _p, _p]),
        "orc_spmv": (None, [_p, _p, _p, _p, _i64, _p]),
        "orc_num_threads": (ctypes.c_int, []),
        "orc_face_normals": (None, [_p, _p, _i64, _p]),
        "orc_neighborhoods": (_i64, [_p, _i64, ctypes.c_int, _p, _p]),
        "orc_rho_tilde_kernel": (None, [_p, _p, _p, _p, _p, _p, _p, _p, _i64, _d, _d, _d, _d, _d,
                                        _d, _d, _d, _p, _p]),
        "orc_rho_tilde_blend": (None, [_p, _p, _p, _p, _p, _p, _p, _i64, _d, _d, _d, _d, _d,
                                       _d, _d, _d, _p, _p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ---------------------------------------------------------------- physics

def q2_at_mach(mach, m_inf, gamma=GAMMA):
    return float(lib().orc_q2_at_mach(mach, m_inf, gamma))


def density_field(q2, m_inf, gamma=GAMMA):
    q2 = _c(q2, np.float64)
    out = np.empty_like(q2)
    lib().orc_density_field(_ptr(q2), q2.size, m_inf, gamma, _ptr(out))
    return out


def mach_squared_field(q2, m_inf, gamma=GAMMA):
    q2 = _c(q2, np.float64)
    out = np.empty_like(q2)
    lib().orc_mach2_field(_ptr(q2), q2.size, m_inf, gamma, _ptr(out))
    return out


def limit_q2_field(q2, m_inf, m_cap, gamma=GAMMA):
    q2 = _c(q2, np.float64)
    out = np.empty_like(q2)
    lib().orc_limit_q2_field(_ptr(q2), q2.size, m_inf, m_cap, gamma, _ptr(out))
    return out


def density_derivative_field(q2, m_inf, gamma=GAMMA):
    q2 = _c(q2, np.float64)
    out = np.empty_like(q2)
    lib().orc_drho_field(_ptr(q2), q2.size, m_inf, gamma, _ptr(out))
    return out


# ------------------------------------------------------------------- mesh

def element_geometry(nodes, elements):
    nodes = _c(nodes, np.float64)
    el = _c(elements, np.int32)
    E = len(el)
    B = np.empty((E, 4, 3))
    V = np.empty(E)
    bad = lib().orc_element_geometry(_ptr(nodes), _ptr(el), E, _ptr(B), _ptr(V))
    if bad >= 0:
        raise ValueError(f"element_gradients: degenerate tetrahedron {bad}")
    return B, V


def face_adjacency(elements):
    el = _c(elements, np.int32)
    fn = np.empty((len(el), 4), dtype=np.int32)
    lib().orc_face_adjacency(_ptr(el), len(el), _ptr(fn))
    return fn


def centroids(nodes, elements):
    nodes = _c(nodes, np.float64)
    el = _c(elements, np.int32)
    out = np.empty((len(el), 3))
    lib().orc_centroids(_ptr(nodes), _ptr(el), len(el), _ptr(out))
    return out


def greedy_coloring(elements, n_nodes):
    el = _c(elements, np.int32)
    colors = np.empty(len(el), dtype=np.int32)
    nc = lib().orc_greedy_coloring(_ptr(el), len(el), n_nodes, _ptr(colors))
    if nc < 0:
        raise ValueError("greedy coloring exceeded 256 colors")
    return colors, int(nc)


def color_partition_csr(elements, n_nodes):
    colors, nc = greedy_coloring(elements, n_nodes)
    off = np.empty(nc + 1, dtype=np.int64)
    elems = np.empty(len(colors), dtype=np.int64)
    lib().orc_color_partition(_ptr(colors), len(colors), nc, _ptr(off), _ptr(elems))
    return off, elems, nc


def csr_pattern(elements, n_nodes):
    el = _c(elements, np.int32)
    indptr = np.empty(n_nodes + 1, dtype=np.int64)
    nnz = lib().orc_csr_pattern(_ptr(el), len(el), n_nodes, _ptr(indptr), None)
    indices = np.empty(nnz, dtype=np.int32)
    lib().orc_csr_pattern(_ptr(el), len(el), n_nodes, _ptr(indptr), _ptr(indices))
    return indptr, indices


def elem_to_csr(elements, indptr, indices):
    el = _c(elements, np.int32)
    indptr = _c(indptr, np.int64)
    indices = _c(indices, np.int32)
    out = np.empty((len(el), 4, 4), dtype=np.int64)
    lib().orc_elem_to_csr(_ptr(el), len(el), _ptr(indptr), _ptr(indices), _ptr(out))
    return out


# -------------------------------------------------------------- operators

class PicardOperator:
    """Oracle restatement of ``kernels/jacobian.py:231-375``."""

    def __init__(self, nodes, elements):
        self.nodes = _c(nodes, np.float64)
        self.elements = _c(elements, np.int32)
        self.n_nodes = len(self.nodes)
        self.n_tets = len(self.elements)
        self.B, self.V = element_geometry(self.nodes, self.elements)
        self.color_offsets, self.color_elems, self.n_colors = color_partition_csr(
            self.elements, self.n_nodes)
        self.indptr, self.indices = csr_pattern(self.elements, self.n_nodes)
        self.nnz = len(self.indices)
        self.elem_to_csr = elem_to_csr(self.elements, self.indptr, self.indices)
        self._grad = np.empty((self.n_tets, 3))
        self._q2 = np.empty(self.n_tets)
        self._R = np.empty(self.n_nodes)
        self.rho_ones = np.ones(self.n_tets)
        self.newton_nnz = None
        self.n_term3_active = None

    def _csr(self, data):
        return sp.csr_matrix((data, self.indices, self.indptr),
                             shape=(self.n_nodes, self.n_nodes))

    def velocities(self, phi):
        phi = _c(phi, np.float64)
        lib().orc_velocities(_ptr(self.elements), _ptr(self.B), _ptr(phi),
                             self.n_tets, _ptr(self._grad), _ptr(self._q2))
        return self._grad, self._q2

    def assemble_matrix(self, rho_tilde=None):
        rt = self.rho_ones if rho_tilde is None else _c(rho_tilde, np.float64)
        data = np.empty(self.nnz)
        lib().orc_matrix_data(_ptr(self.color_offsets), _ptr(self.color_elems),
                              self.n_colors, _ptr(self.elem_to_csr), _ptr(self.B),
                              _ptr(self.V), _ptr(rt), self.nnz, _ptr(data))
        return self._csr(data)

    def assemble_residual(self, phi, rho_tilde=None):
        rt = self.rho_ones if rho_tilde is None else _c(rho_tilde, np.float64)
        grad, _ = self.velocities(phi)
        lib().orc_residual(_ptr(self.color_offsets), _ptr(self.color_elems),
                           self.n_colors, _ptr(self.elements), _ptr(self.B),
                           _ptr(self.V), _ptr(rt), _ptr(grad), self.n_nodes,
                           _ptr(self._R))
        return self._R

    def assemble_newton_jacobian(self, phi, rho_tilde, s_e, s_u, upstream,
                                 u_inf=1.0, lim_mask=None):
        upstream = _c(upstream, np.int64)
        if lim_mask is not None:
            s_e = s_e * lim_mask
            s_u = s_u * lim_mask[upstream]
        s_e = _c(s_e, np.float64)
        s_u = _c(s_u, np.float64)
        rt = _c(rho_tilde, np.float64)
        inv_u2 = 1.0 / (u_inf * u_inf)
        phi = _c(phi, np.float64)
        grad = np.empty((self.n_tets, 3))
        q2 = np.empty(self.n_tets)
        lib().orc_velocities(_ptr(self.elements), _ptr(self.B), _ptr(phi),
                             self.n_tets, _ptr(grad), _ptr(q2))
        data = np.empty(self.nnz)
        lib().orc_jacobian_data(_ptr(self.color_offsets), _ptr(self.color_elems),
                                self.n_colors, _ptr(self.elem_to_csr), _ptr(self.B),
                                _ptr(self.V), _ptr(rt), _ptr(grad), _ptr(s_e),
                                inv_u2, self.nnz, _ptr(data))
        J = self._csr(data)
        active = np.nonzero(s_u)[0].astype(np.int64)
        self.n_term3_active = int(len(active))
        if len(active) > 0:
            n = 16 * len(active)
            rows = np.empty(n, dtype=np.int64)
            cols = np.empty(n, dtype=np.int64)
            vals = np.empty(n)
            lib().orc_term3_coo(_ptr(active), len(active), _ptr(self.elements),
                                _ptr(self.B), _ptr(self.V), _ptr(grad), _ptr(upstream),
                                _ptr(s_u), inv_u2, _ptr(rows), _ptr(cols), _ptr(vals))
            J = (J + sp.coo_matrix((vals, (rows, cols)), shape=J.shape).tocsr()).tocsr()
        self.newton_nnz = int(J.nnz)
        return J


def face_normals(nodes, elements):
    """compute_face_normals (kernels/upwind.py:128-172): (n, 4, 3)."""
    X, el = _c(nodes, np.float64), _c(elements, np.int32)
    out = np.empty((len(el), 4, 3))
    lib().orc_face_normals(_ptr(X), _ptr(el), len(el), _ptr(out))
    return out


def build_upstream_neighborhoods(face_neighbors, depth=3):
    """build_upstream_neighborhoods (kernels/upwind.py:313-341): CSR
    (offsets int64, indices int64) of the elements within `depth` face
    hops, e excluded, ascending."""
    fn = _c(face_neighbors, np.int32)
    n = len(fn)
    off = np.zeros(n + 1, dtype=np.int64)
    total = lib().orc_neighborhoods(_ptr(fn), n, int(depth), _ptr(off), None)
    idx = np.empty(max(total, 1), dtype=np.int32)
    lib().orc_neighborhoods(_ptr(fn), n, int(depth), _ptr(off), _ptr(idx))
    return off, idx[:total].astype(np.int64)


class UpwindOperator:
    """Oracle restatement of ``kernels/upwind.py:733-920``: the walk flux,
    and the weighted "kernel" / "blend" modes of ``rho_tilde``."""

    def __init__(self, nodes, elements, weighted=False, mode="kernel", p_weight=3.0,
                 reach_frac=1.0, reach_gain_max=4.0, nbr_depth=3, sigma_s_frac=0.35,
                 sigma_p_frac=0.35):
        self.nodes = _c(nodes, np.float64)
        self.elements = _c(elements, np.int32)
        self.face_neighbors = face_adjacency(self.elements)
        self.centroids = centroids(self.nodes, self.elements)
        self.weighted, self.mode = weighted, mode
        self.p_weight, self.reach_frac, self.reach_gain_max = p_weight, reach_frac, reach_gain_max
        self.sigma_s_frac, self.sigma_p_frac = sigma_s_frac, sigma_p_frac
        self._nb_off = self._nb_idx = None
        if weighted and mode == "kernel":
            self._nb_off, self._nb_idx = build_upstream_neighborhoods(self.face_neighbors, nbr_depth)
        n = len(self.elements)
        self._upstream = np.empty(n, dtype=np.int64)
        self.nu = np.empty(n)
        self._rho_tilde = np.empty(n)
        self._se = np.empty(n)
        self._su = np.empty(n)
        self._branch = np.empty(n, dtype=np.int8)
        self.nu_max = 0.0
        self.n_supersonic = 0
        self.n_floored = 0

    def upstream(self, grad, max_hops=4):
        grad = _c(grad, np.float64)
        fn = _c(self.face_neighbors, np.int32)
        lib().orc_upstream(_ptr(fn), _ptr(self.centroids), _ptr(self.nodes),
                           _ptr(self.elements), _ptr(grad), len(self.elements),
                           max_hops, _ptr(self._upstream))
        return self._upstream

    def _monitors(self, rho_floor, branch=None):
        self.nu_max = float(self.nu.max())
        self.n_supersonic = int(np.count_nonzero(self.nu > 0.0))
        if branch is None:
            self.n_floored = int(np.count_nonzero(self._rho_tilde == rho_floor))
        else:
            self.n_floored = int(np.count_nonzero(branch == 3))

    def rho_tilde(self, grad, q2, rho, m_inf, C, m_crit, gamma=GAMMA, rho_floor=0.05):
        if self.weighted:
            return self._rho_tilde_weighted(grad, q2, rho, m_inf, C, m_crit, gamma, rho_floor)
        up = self.upstream(grad)
        q2, rho = _c(q2, np.float64), _c(rho, np.float64)
        lib().orc_rho_tilde(_ptr(q2), _ptr(rho), _ptr(up), len(q2), m_inf, m_crit, C,
                            gamma, rho_floor, _ptr(self.nu), _ptr(self._rho_tilde))
        self._monitors(rho_floor)
        return self._rho_tilde

    def _rho_tilde_weighted(self, grad, q2, rho, m_inf, C, m_crit, gamma, rho_floor):
        grad = _c(grad, np.float64)
        q2, rho = _c(q2, np.float64), _c(rho, np.float64)
        cen = _c(self.centroids, np.float64)
        n = len(q2)
        if self.mode == "kernel":
            off = _c(self._nb_off, np.int64)
            idx = _c(self._nb_idx, np.int32)
            lib().orc_rho_tilde_kernel(_ptr(q2), _ptr(rho), _ptr(grad), _ptr(self.nodes),
                                       _ptr(self.elements), _ptr(cen), _ptr(off), _ptr(idx), n,
                                       m_inf, m_crit, C, gamma, rho_floor, self.reach_frac,
                                       self.sigma_s_frac, self.sigma_p_frac, _ptr(self.nu),
                                       _ptr(self._rho_tilde))
        else:
            fn = _c(self.face_neighbors, np.int32)
            lib().orc_rho_tilde_blend(_ptr(q2), _ptr(rho), _ptr(grad), _ptr(self.nodes),
                                      _ptr(self.elements), _ptr(cen), _ptr(fn), n, m_inf, m_crit, C,
                                      gamma, rho_floor, self.p_weight, self.reach_frac,
                                      self.reach_gain_max, _ptr(self.nu), _ptr(self._rho_tilde))
        self._monitors(rho_floor)
        return self._rho_tilde

    def freeze_upwind_state(self, grad, q2, rho, m_inf, C, m_crit, gamma=GAMMA,
                            rho_floor=0.05):
        up = self.upstream(grad)
        q2, rho = _c(q2, np.float64), _c(rho, np.float64)
        lib().orc_classify(_ptr(q2), _ptr(rho), _ptr(up), len(q2), m_inf, m_crit, C,
                           gamma, rho_floor, _ptr(self._branch))
        return up.copy(), self._branch.copy()

    def rho_tilde_frozen(self, q2, rho, upstream, branch, m_inf, C, m_crit,
                         gamma=GAMMA, rho_floor=0.05):
        q2, rho = _c(q2, np.float64), _c(rho, np.float64)
        up, br = _c(upstream, np.int64), _c(branch, np.int8)
        lib().orc_rho_tilde_frozen(_ptr(q2), _ptr(rho), _ptr(up), _ptr(br), len(q2),
                                   m_inf, m_crit, C, gamma, rho_floor, _ptr(self.nu),
                                   _ptr(self._rho_tilde))
        self._monitors(rho_floor, branch=br)
        return self._rho_tilde

    def rho_tilde_frozen_sensitivities(self, q2, rho, upstream, branch, m_inf, C,
                                       m_crit, gamma=GAMMA, rho_floor=0.05):
        q2, rho = _c(q2, np.float64), _c(rho, np.float64)
        up, br = _c(upstream, np.int64), _c(branch, np.int8)
        lib().orc_sens_frozen(_ptr(q2), _ptr(rho), _ptr(up), _ptr(br), len(q2), m_inf,
                              m_crit, C, gamma, rho_floor, _ptr(self._se), _ptr(self._su))
        return self._se, self._su

    def rho_tilde_sensitivities(self, grad, q2, rho, m_inf, C, m_crit, gamma=GAMMA,
                                rho_floor=0.05):
        up = self.upstream(grad)
        q2, rho = _c(q2, np.float64), _c(rho, np.float64)
        lib().orc_sens(_ptr(q2), _ptr(rho), _ptr(up), len(q2), m_inf, m_crit, C, gamma,
                       rho_floor, _ptr(self._se), _ptr(self._su))
        return self._se, self._su, self._upstream


def spmv(indptr, indices, data, x):
    indptr, indices = _c(indptr, np.int64), _c(indices, np.int32)
    data, x = _c(data, np.float64), _c(x, np.float64)
    y = np.empty(len(indptr) - 1)
    lib().orc_spmv(_ptr(indptr), _ptr(indices), _ptr(data), _ptr(x), len(y), _ptr(y))
    return y


# ------------------------------------------------------------------ chain

M_CRIT = 0.95
UPWIND_C = 1.5
RHO_FLOOR = 0.05
M_CAP = 3.0


def chain(op: PicardOperator, upw: UpwindOperator, phi, m_inf, u_inf=1.0,
          m_cap=M_CAP, C=UPWIND_C, m_crit=M_CRIT, rho_floor=RHO_FLOOR,
          gamma=GAMMA, jacobian=True):
    """Residual + Jacobian at phi, composed like eval_residual and
    assemble_coupled (pyfp3d/solve/newton.py:345-372, :435-452)."""
    out = {}
    grad, q2 = op.velocities(phi)
    grad, q2 = grad.copy(), q2.copy()
    q2n = q2 / u_inf ** 2
    q2l = limit_q2_field(q2n, m_inf, m_cap, gamma)
    lim = q2l == q2n
    rho = density_field(q2l, m_inf, gamma)
    rt = upw.rho_tilde(grad, q2l, rho, m_inf, C, m_crit, gamma, rho_floor).copy()
    out.update(grad=grad, q2=q2, q2l=q2l, lim=lim, rho=rho, rho_tilde=rt,
               nu=upw.nu.copy(), upstream=upw._upstream.copy(),
               nu_max=upw.nu_max, n_supersonic=upw.n_supersonic,
               n_floored=upw.n_floored, n_limited=int(np.count_nonzero(~lim)))
    out["R"] = op.assemble_residual(phi, rt).copy()
    if jacobian:
        s_e, s_u, up = upw.rho_tilde_sensitivities(grad, q2l, rho, m_inf, C, m_crit,
                                                   gamma, rho_floor)
        s_e, s_u, up = s_e.copy(), s_u.copy(), up.copy()
        J = op.assemble_newton_jacobian(phi, rt, s_e, s_u, up, u_inf=u_inf,
                                        lim_mask=None if lim.all() else lim)
        out.update(s_e=s_e, s_u=s_u, J=J, n_term3_active=op.n_term3_active,
                   newton_nnz=op.newton_nnz)
    return out


class WakeConstraint:
    """Oracle restatement of the wake master-slave elimination
    (``constraints/wake.py:32-127``): T maps every cut-mesh node to its
    reduced node (a slave to its master), A_red = T^T A T, H = T^T A G with
    G the per-station slave indicators, h = H^T as a dense array."""

    def __init__(self, A, wc):
        n_cut, n_red, n_dup = A.shape[0], wc.n_nodes_orig, len(wc.slave_nodes)
        if n_cut != n_red + n_dup:
            raise ValueError(f"A is {n_cut}x{n_cut} but WakeCut implies {n_red} + {n_dup} nodes")
        red = np.arange(n_cut, dtype=np.int64)
        red[np.asarray(wc.slave_nodes, dtype=np.int64)] = np.asarray(wc.master_nodes, dtype=np.int64)
        self.T = sp.csr_matrix((np.ones(n_cut), (np.arange(n_cut), red)), shape=(n_cut, n_red))
        self.wc, self.n_reduced = wc, n_red
        self.update_matrix(A)

    def reduce_operator(self, A):
        A = sp.csr_matrix(A)
        wc = self.wc
        G = sp.csr_matrix((np.ones(len(wc.slave_nodes)), (np.asarray(wc.slave_nodes), np.asarray(wc.node_station))),
                          shape=(self.T.shape[0], wc.n_stations))
        A_red = (self.T.T @ (A @ self.T)).tocsr()
        H = (self.T.T @ (A @ G)).tocsr()
        for M in (A_red, H):
            M.sum_duplicates()
            M.sort_indices()
        return A_red, H

    def update_matrix(self, A):
        self.A_reduced, H = self.reduce_operator(A)
        self._h = H.T.toarray()

    def reduced_rhs(self, b, gamma):
        gamma = np.atleast_1d(np.asarray(gamma, dtype=np.float64))
        return self.T.T @ np.asarray(b, dtype=np.float64) - gamma @ self._h

    def expand(self, phi_red, gamma):
        wc = self.wc
        phi = np.empty(self.n_reduced + len(wc.slave_nodes))
        phi[:self.n_reduced] = phi_red
        phi[wc.slave_nodes] = np.asarray(phi_red)[wc.master_nodes] + wc.gamma_at_nodes(gamma)
        return phi


def kutta_targets(phi, wc):
    """Per-station mean of phi[upper probe] - phi[lower probe]
    (``constraints/wake.py:196-212``)."""
    jumps = np.asarray(phi)[wc.kutta_upper] - np.asarray(phi)[wc.kutta_lower]
    sums = np.bincount(wc.te_station, weights=jumps, minlength=wc.n_stations)
    return sums / np.bincount(wc.te_station, minlength=wc.n_stations)


# -------------------------------------------------- coupled (phi, Gamma) Newton
# solve/newton.py:97-1141 restated for the probe Kutta estimator, with the
# far-field split and basis given (dir_red, vals0_red, V_red: set_mach's
# output) and exact (sparse LU + Woodbury) Newton steps -- the reference's
# precond="direct" path (:966-1011).


class LiftingSystem:
    """NewtonWorkspace.eval_residual / assemble_coupled / the probe
    kutta_blocks (solve/newton.py:326-502) over the oracle kernels."""

    def __init__(self, nodes, elements, wc, dir_red, vals0_red, V_red, tip_taper=None, u_inf=1.0,
                 external_rhs=None):
        self.op = PicardOperator(nodes, elements)
        self.upw = UpwindOperator(nodes, elements)
        self.wc, self.u_inf = wc, float(u_inf)
        self.con = WakeConstraint(self.op.assemble_matrix(np.ones(len(elements))), wc)
        self.n_red, self.n_st = self.con.n_reduced, wc.n_stations
        self.dir_red = np.asarray(dir_red, dtype=np.int64)
        is_dir = np.zeros(self.n_red, dtype=bool)
        is_dir[self.dir_red] = True
        self.free = np.where(~is_dir)[0]
        self.vals0_red, self.V_red = np.asarray(vals0_red), np.asarray(V_red)
        self.taper = np.ones(self.n_st) if tip_taper is None else np.asarray(tip_taper, dtype=np.float64)
        self.b_ext = None if external_rhs is None else np.asarray(external_rhs, dtype=np.float64)
        counts = np.bincount(wc.te_station, minlength=self.n_st).astype(np.float64)
        probes = np.concatenate([wc.kutta_upper, wc.kutta_lower])
        cols = np.searchsorted(self.free, probes)
        w = 1.0 / counts[wc.te_station]
        self.K = sp.coo_matrix((np.concatenate([w, -w]), (np.concatenate([wc.te_station, wc.te_station]), cols)),
                               shape=(self.n_st, len(self.free))).tocsr()
        if not np.all(self.taper == 1.0):
            self.K = sp.diags(self.taper) @ self.K

    def eval_residual(self, phi_free, gamma, m_inf, frozen=None, **kw):
        """(R_free, F, state) (newton.py:340-419)."""
        gamma = np.asarray(gamma, dtype=np.float64)
        phi_red = np.empty(self.n_red)
        phi_red[self.free] = phi_free
        phi_red[self.dir_red] = self.vals0_red + self.V_red @ gamma
        phi_cut = self.con.expand(phi_red, gamma)
        st = chain(self.op, self.upw, phi_cut, m_inf, self.u_inf, jacobian=True, **kw)
        R_red = self.con.T.T @ (st["R"] if self.b_ext is None else st["R"] - self.b_ext)
        F = self.taper * kutta_targets(phi_cut, self.wc) - gamma
        st.update(phi_red=phi_red, phi_cut=phi_cut)
        return R_red[self.free], F, st

    def blocks(self, st):
        """(J_ff, B), B = J_red[free, dir] V + H_J[free] (newton.py:430-457)."""
        J_red, H = self.con.reduce_operator(st["J"])
        J_ff = J_red[self.free][:, self.free].tocsr()
        J_fd = J_red[self.free][:, self.dir_red].tocsr()
        B = J_fd @ sp.csr_matrix(self.V_red) + H.tocsr()[self.free, :]
        return J_ff, B.tocsc()

    def solve(self, phi_free, gamma, m_inf, n_newton_max=30, tol_residual=1e-10, tol_gamma=1e-8, **kw):
        """Exact Newton with the merit line search (newton.py:779-1111 on
        the precond="direct" branch, live upwind selection):
        (phi_cut, gamma, residual history)."""
        import scipy.sparse.linalg as spla
        phi_free = np.asarray(phi_free, dtype=np.float64).copy()
        gamma = np.asarray(gamma, dtype=np.float64).copy()
        R, F, st = self.eval_residual(phi_free, gamma, m_inf, **kw)
        merit = float(R @ R + F @ F)
        hist = []
        for _ in range(n_newton_max):
            r_norm = float(np.max(np.abs(R)))
            hist.append(r_norm)
            if (np.max(np.abs(F)) < tol_gamma and st["n_limited"] == 0 and st["n_floored"] == 0
                    and r_norm < tol_residual):
                return st["phi_cut"], gamma, hist, True
            J_ff, B = self.blocks(st)
            rhs = -R - B @ F
            lu = spla.splu(J_ff.tocsc())
            z = lu.solve(rhs)
            JB = lu.solve(B.toarray())
            S = np.eye(self.n_st) + self.K @ JB
            dphi = z - JB @ np.linalg.solve(S, self.K @ z)
            dgamma = self.K @ dphi + F
            lam, best = 1.0, None
            for _ in range(5):
                R_t, F_t, st_t = self.eval_residual(phi_free + lam * dphi, gamma + lam * dgamma, m_inf, **kw)
                m_t = float(R_t @ R_t + F_t @ F_t)
                if np.isfinite(m_t) and m_t <= merit:
                    best = None
                    break
                if np.isfinite(m_t) and (best is None or m_t < best[0]):
                    best = (m_t, lam, R_t, F_t, st_t)
                lam *= 0.5
            if best is not None:
                m_t, lam, R_t, F_t, st_t = best
            phi_free = phi_free + lam * dphi
            gamma = gamma + lam * dgamma
            R, F, st, merit = R_t, F_t, st_t, m_t
        return st["phi_cut"], gamma, hist, False


# ---------------------------------------------------------------- wall post
# post/surface.py:80-363, restated with numpy (the per-triangle arithmetic
# in the reference's order).

def _cross(a, b):
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                     a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1)


def _dot(a, b):
    return (a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1]) + a[:, 2] * b[:, 2]


def wall_tri_gradients(nodes, wall_faces, phi):
    """In-plane P1 gradient, area and stored-winding unit normal of each wall
    triangle (post/surface.py:80-118)."""
    wf = np.asarray(wall_faces, dtype=np.int64)
    p0, p1, p2 = nodes[wf[:, 0]], nodes[wf[:, 1]], nodes[wf[:, 2]]
    ed1, ed2 = p1 - p0, p2 - p0
    av = _cross(ed1, ed2)
    ta = np.sqrt(_dot(av, av))
    tn = av / ta[:, None]
    e1 = ed1 / np.sqrt(_dot(ed1, ed1))[:, None]
    e2 = _cross(tn, e1)
    u1, v1, u2, v2 = _dot(ed1, e1), _dot(ed1, e2), _dot(ed2, e1), _dot(ed2, e2)
    phi = np.asarray(phi)
    df1, df2 = phi[wf[:, 1]] - phi[wf[:, 0]], phi[wf[:, 2]] - phi[wf[:, 0]]
    det = u1 * v2 - v1 * u2
    du = (v2 * df1 - v1 * df2) / det
    dv = (-u2 * df1 + u1 * df2) / det
    return du[:, None] * e1 + dv[:, None] * e2, 0.5 * ta, tn


def wall_owners(elements, wall_faces):
    """The one tet owning each wall triangle (ValueError otherwise)."""
    el = np.asarray(elements, dtype=np.int64)
    faces = np.concatenate([el[:, [1, 2, 3]], el[:, [0, 2, 3]], el[:, [0, 1, 3]], el[:, [0, 1, 2]]])
    faces.sort(axis=1)
    owner_of = {}
    for i, f in enumerate(map(tuple, faces)):
        owner_of.setdefault(f, []).append(i % len(el))
    out = []
    for f in map(tuple, np.sort(np.asarray(wall_faces, dtype=np.int64), axis=1)):
        own = owner_of.get(f, [])
        if len(own) != 1:
            raise ValueError("wall face not owned by exactly one tet")
        out.append(own[0])
    return np.array(out, dtype=np.int64)


def wall_outward_normals(nodes, elements, wall_faces):
    """Unit normals pointing toward the owning tet (post/surface.py:192-231)."""
    wf = np.asarray(wall_faces, dtype=np.int64)
    owner = wall_owners(elements, wf)
    _, _, n = wall_tri_gradients(nodes, wf, np.zeros(len(nodes)))
    fc = ((nodes[wf[:, 0]] + nodes[wf[:, 1]]) + nodes[wf[:, 2]]) / 3.0
    el = np.asarray(elements, dtype=np.int64)[owner]
    oc = (((nodes[el[:, 0]] + nodes[el[:, 1]]) + nodes[el[:, 2]]) + nodes[el[:, 3]]) / 4.0
    n = n.copy()
    n[_dot(n, oc - fc) < 0] *= -1.0
    return n


def wall_adjacency(wall_faces):
    """Edge neighbour of each triangle across edges (0,1), (1,2), (2,0), -1
    on a boundary edge or an edge of more than two triangles
    (post/surface.py:121-144)."""
    wf = np.asarray(wall_faces, dtype=np.int64)
    adj = np.full((len(wf), 3), -1, dtype=np.int64)
    occ = {}
    for t in range(len(wf)):
        for k, (a, b) in enumerate(((0, 1), (1, 2), (2, 0))):
            va, vb = wf[t, a], wf[t, b]
            occ.setdefault((min(va, vb), max(va, vb)), []).append((t, k))
    for v in occ.values():
        if len(v) == 2:
            (t0, k0), (t1, k1) = v
            adj[t0, k0], adj[t1, k1] = t1, t0
    return adj


def wall_force_coefficients(nodes, elements, wall_faces, phi, alpha_deg=0.0, u_inf=1.0, s_ref=1.0,
                            m_inf=0.0, smooth_passes=0, gamma=GAMMA):
    """Pressure-integrated force coefficients on the wall
    (post/surface.py:309-363, smoothing :147-189)."""
    g, area, _ = wall_tri_gradients(nodes, wall_faces, phi)
    n_out = wall_outward_normals(nodes, elements, wall_faces)
    if smooth_passes > 0:
        adj = wall_adjacency(wall_faces)
        for _ in range(smooth_passes):
            acc = g * area[:, None]
            wsum = area.copy()
            for k in range(3):
                nb = adj[:, k]
                m = nb >= 0
                m[m] = _dot(n_out[m], n_out[nb[m]]) > 0.2
                acc[m] += g[nb[m]] * area[nb[m], None]
                wsum[m] += area[nb[m]]
            g = acc / wsum[:, None]
    q2 = _dot(g, g) / u_inf ** 2
    if m_inf > 0.0:
        base = np.maximum(1.0 + 0.5 * (gamma - 1.0) * (m_inf * m_inf) * (1.0 - q2), 1e-10)
        rho = base ** (1.0 / (gamma - 1.0))
        cp = 2.0 / (gamma * m_inf ** 2) * (rho ** gamma - 1.0)
    else:
        cp = 1.0 - q2
    cf = -((cp * area)[:, None] * n_out).sum(axis=0) / s_ref
    a = np.deg2rad(alpha_deg)
    lift, drag = np.array([-np.sin(a), np.cos(a), 0.0]), np.array([np.cos(a), np.sin(a), 0.0])
    return {"cl": float(cf @ lift), "cd_pressure": float(cf @ drag), "cf": cf, "cp_tri": cp}


def newton_terms23_side_coo(B, V, side, u_inf=1.0):
    """Per-side Newton Terms 2 and 3 as COO triplets on extended DOFs
    (kernels/cut_assembly.py:401-488): rows from the residual DOF map,
    columns from the read map; Term-2 blocks of the kept elements with
    s_e != 0 (ascending), then Term-3 blocks of those with s_u != 0."""
    B = np.asarray(B).reshape(-1, 4, 3)
    keep, dof = np.asarray(side["keep"]), np.asarray(side["dofvec"], dtype=np.int64)
    read = np.asarray(side.get("readvec", dof), dtype=np.int64)
    grad = np.asarray(side["grad"])
    grad_row = np.asarray(side.get("grad_row", grad))
    lim = np.asarray(side["lim_mask"])
    inv_u2 = 1.0 / (u_inf * u_inf)
    gbr = ((grad_row[:, None, 0] * B[:, :, 0] + grad_row[:, None, 1] * B[:, :, 1])
           + grad_row[:, None, 2] * B[:, :, 2])
    gb = (grad[:, None, 0] * B[:, :, 0] + grad[:, None, 1] * B[:, :, 1]) + grad[:, None, 2] * B[:, :, 2]
    up = np.asarray(side["upstream"], dtype=np.int64)
    s_e = np.asarray(side["s_e"]) * lim
    s_u = np.asarray(side["s_u"]) * lim[up]
    rows, cols, data = [], [], []
    e2 = np.flatnonzero(keep & (s_e != 0.0))
    w2 = (2.0 * inv_u2) * s_e[e2] * V[e2]
    rows.append(np.repeat(dof[e2], 4, axis=1).reshape(-1))
    cols.append(np.tile(read[e2], (1, 4)).reshape(-1))
    data.append((w2[:, None, None] * (gbr[e2][:, :, None] * gb[e2][:, None, :])).reshape(-1))
    e3 = np.flatnonzero(keep & (s_u != 0.0))
    u3 = up[e3]
    w3 = (2.0 * inv_u2) * s_u[e3] * V[e3]
    rows.append(np.repeat(dof[e3], 4, axis=1).reshape(-1))
    cols.append(np.tile(read[u3], (1, 4)).reshape(-1))
    data.append((w3[:, None, None] * (gbr[e3][:, :, None] * gb[u3][:, None, :])).reshape(-1))
    return np.concatenate(rows), np.concatenate(cols), np.concatenate(data)
