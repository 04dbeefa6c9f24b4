"""UpwindOperator on the B200: the multi-hop upstream walk, the upwinded
density and its exact sensitivities, live and frozen, and the weighted
"kernel" / "blend" densities, with the reference's signatures
(pyfp3d/kernels/upwind.py:128-454, :733-920).

Arrays in, same kind out (numpy -> numpy host copies, CUDA tensors -> device
views into the workspace).  The monitors nu_max / n_supersonic / n_floored
are read from the device on first access after each sweep.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .. import _lib as L
from ..mesh.device import get_mesh
from ..physics.isentropic import GAMMA


def compute_face_normals(nodes, elements, out) -> None:
    """Outward unit normal of each face, face f opposite local node f, into
    `out` (n_tets, 4, 3) (kernels/upwind.py:128-172)."""
    mesh = get_mesh(nodes, elements)
    d = L.torch().empty((mesh.n_tets, 4, 3), dtype=L.torch().float64, device="cuda")
    L.call("up3d_face_normals", mesh.handle, d.data_ptr(), L.stream_ptr())
    if L.is_torch(out):
        out.copy_(d)
    else:
        out[...] = d.cpu().numpy()


def build_upstream_neighborhoods(face_neighbors, depth: int = 3):
    """The elements within `depth` face hops of each element, itself
    excluded, ascending, as CSR (offsets, indices) int64
    (kernels/upwind.py:313-341).  Any depth >= 1 (deeper than 4 hops built on the host)."""
    t = L.torch()
    fn = L.to_device(face_neighbors, t.int32)
    n = int(fn.shape[0])
    off = t.empty(n + 1, dtype=t.int64, device="cuda")
    total = ctypes.c_int64()
    L.call("up3d_face_neighborhoods", fn.data_ptr(), n, int(depth), off.data_ptr(), None,
           ctypes.byref(total), L.stream_ptr())
    idx = t.empty(max(total.value, 1), dtype=t.int32, device="cuda")
    L.call("up3d_face_neighborhoods", fn.data_ptr(), n, int(depth), off.data_ptr(), idx.data_ptr(),
           ctypes.byref(total), L.stream_ptr())
    idx = idx[:total.value].to(t.int64)
    if L.is_torch(face_neighbors):
        return off, idx
    return off.cpu().numpy(), idx.cpu().numpy()


class UpwindOperator:
    """B200 UpwindOperator (kernels/upwind.py:733-920): the walk flux, or
    with weighted=True the streamline-kernel (mode "kernel") or face-blend
    (any other mode) density; the weighted modes offer rho_tilde only, as
    the reference's do."""

    def __init__(self, nodes, elements, weighted: bool = False, mode: str = "kernel",
                 p_weight: float = 3.0, reach_frac: float = 1.0, reach_gain_max: float = 4.0,
                 nbr_depth: int = 3, sigma_s_frac: float = 0.35, sigma_p_frac: float = 0.35, *, mesh=None):
        # mesh (keyword only, not in the reference's signature): a DeviceMesh
        # of these nodes and elements instead of the shared handle
        t = L.require_cuda()
        self._mesh = mesh if mesh is not None else get_mesh(nodes, elements)
        self._host = not L.is_torch(nodes)
        self.weighted = bool(weighted)
        self.mode = mode
        self.nbr_depth = int(nbr_depth)
        self._nb = None
        if self.weighted and mode == "kernel":
            self._neighborhoods()
        self.p_weight, self.reach_frac, self.reach_gain_max = p_weight, reach_frac, reach_gain_max
        self.sigma_s_frac, self.sigma_p_frac = sigma_s_frac, sigma_p_frac
        self._nodes = self._mesh.nodes
        self._elements = self._mesh.elements
        E = self._mesh.n_tets
        self._upstream_d = t.empty(E, dtype=t.int64, device="cuda")
        self._nu_d = t.empty(E, dtype=t.float64, device="cuda")
        self._rt_d = t.empty(E, dtype=t.float64, device="cuda")
        self._se_d = t.empty(E, dtype=t.float64, device="cuda")
        self._su_d = t.empty(E, dtype=t.float64, device="cuda")
        self._branch_d = t.empty(E, dtype=t.int8, device="cuda")
        self._mon = L.monitors_buffer()
        self._mon_cache = {"nu_max": 0.0, "n_supersonic": 0, "n_floored": 0}
        self._mon_dirty = False
        self._upstream = np.empty(E, dtype=np.int64)
        self._nu = np.empty(E)
        self._rho_tilde = np.empty(E)
        self._se = np.empty(E)
        self._su = np.empty(E)
        self._branch = np.empty(E, dtype=np.int8)
        self._fn = None
        self._cen = None

    # ---------------------------------------------------------- attributes

    @property
    def face_neighbors(self):
        if self._fn is None:
            d = self._mesh.face_neighbors()
            self._fn = d.cpu().numpy() if self._host else d
        return self._fn

    @face_neighbors.setter
    def face_neighbors(self, value):
        # The per-side masking of the level-set path assigns a new array
        # (wake/multivalued.py:463-467); the walk reads the device copy.
        # A masked copy lives on this operator only: the shared mesh
        # handle is forked first.
        from ..mesh.device import DeviceMesh
        self._mesh = DeviceMesh(self._mesh.nodes, self._mesh.elements, self._mesh.device)
        self._mesh.set_face_neighbors(value)
        self._fn = value

    def _neighborhoods(self):
        """The mesh's depth-hop neighbourhood CSR (device views)."""
        off, idx, total = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int64()
        L.call("up3d_mesh_neighborhoods", self._mesh.handle, self.nbr_depth, ctypes.byref(off),
               ctypes.byref(idx), ctypes.byref(total), L.stream_ptr())
        self._nb = (off.value, idx.value, int(total.value))
        return self._nb

    @property
    def _nb_off(self):
        if not (self.weighted and self.mode == "kernel"):
            return None
        from ..mesh.device import device_view
        off = device_view(self._neighborhoods()[0], (self._mesh.n_tets + 1,), np.int64).clone()
        return off.cpu().numpy() if self._host else off

    @property
    def _nb_idx(self):
        if not (self.weighted and self.mode == "kernel"):
            return None
        from ..mesh.device import device_view
        _, ptr, total = self._neighborhoods()
        idx = device_view(ptr, (total,), np.int32).to(L.torch().int64)
        return idx.cpu().numpy() if self._host else idx

    @property
    def centroids(self):
        if self._cen is None:
            d = self._mesh.centroids()
            self._cen = d.cpu().numpy() if self._host else d
        return self._cen

    def _refresh(self):
        if self._mon_dirty:
            m = L.read_monitors(self._mon)
            self._mon_cache = {"nu_max": float(m["nu_max"]),
                               "n_supersonic": int(m["n_supersonic"]),
                               "n_floored": int(m["n_floored"])}
            self._mon_dirty = False
        return self._mon_cache

    @property
    def nu_max(self):
        return self._refresh()["nu_max"]

    @property
    def n_supersonic(self):
        return self._refresh()["n_supersonic"]

    @property
    def n_floored(self):
        return self._refresh()["n_floored"]

    @property
    def nu(self):
        return self._nu_d if not self._host else self._host_copy(self._nu_d, self._nu)

    # ---------------------------------------------------------- helpers

    @staticmethod
    def _host_copy(dev, host):
        host[...] = dev.cpu().numpy()
        return host

    def _flow(self, m_inf, C, m_crit, gamma, rho_floor):
        return L.flow(m_inf, gamma=gamma, m_crit=m_crit, upwind_c=C, rho_floor=rho_floor)

    def _walk(self, grad):
        t = L.torch()
        d_grad = L.to_device(grad, t.float64)
        L.call("up3d_upwind_walk", self._mesh.handle, d_grad.data_ptr(), self._upstream_d.data_ptr(),
               L.stream_ptr())

    def _state(self, q2, rho):
        t = L.torch()
        return L.to_device(q2, t.float64), L.to_device(rho, t.float64)

    # ---------------------------------------------------------- sweeps

    def upstream(self, grad):
        """u(e) of the multi-hop walk (kernels/upwind.py:69-125)."""
        self._walk(grad)
        if L.is_torch(grad):
            return self._upstream_d
        return self._host_copy(self._upstream_d, self._upstream)

    def rho_tilde(self, grad, q2, rho, m_inf, C, m_crit, gamma=GAMMA, rho_floor=0.05):
        """Upwinded densities (kernels/upwind.py:783-819)."""
        if self.weighted:
            return self._rho_tilde_weighted(grad, q2, rho, m_inf, C, m_crit, gamma, rho_floor)
        self._walk(grad)
        d_q2, d_rho = self._state(q2, rho)
        f = self._flow(m_inf, C, m_crit, gamma, rho_floor)
        L.call("up3d_rho_tilde", d_q2.data_ptr(), d_rho.data_ptr(), self._upstream_d.data_ptr(),
               self._mesh.n_tets, f, self._nu_d.data_ptr(), self._rt_d.data_ptr(),
               self._mon.data_ptr(), L.stream_ptr())
        self._mon_dirty = True
        if L.is_torch(q2):
            return self._rt_d
        self._host_copy(self._upstream_d, self._upstream)
        return self._host_copy(self._rt_d, self._rho_tilde)

    def _rho_tilde_weighted(self, grad, q2, rho, m_inf, C, m_crit, gamma, rho_floor):
        """rho_tilde_kernel_sweep / rho_tilde_weighted_sweep
        (kernels/upwind.py:345-454, :176-309)."""
        t = L.torch()
        d_grad = L.to_device(grad, t.float64)
        d_q2, d_rho = self._state(q2, rho)
        f = self._flow(m_inf, C, m_crit, gamma, rho_floor)
        if self.mode == "kernel":
            L.call("up3d_rho_tilde_kernel", self._mesh.handle, d_grad.data_ptr(), d_q2.data_ptr(),
                   d_rho.data_ptr(), f, self.nbr_depth, float(self.reach_frac), float(self.sigma_s_frac),
                   float(self.sigma_p_frac), self._nu_d.data_ptr(), self._rt_d.data_ptr(),
                   self._mon.data_ptr(), L.stream_ptr())
        else:
            L.call("up3d_rho_tilde_blend", self._mesh.handle, d_grad.data_ptr(), d_q2.data_ptr(),
                   d_rho.data_ptr(), f, float(self.p_weight), float(self.reach_frac),
                   float(self.reach_gain_max), self._nu_d.data_ptr(), self._rt_d.data_ptr(),
                   self._mon.data_ptr(), L.stream_ptr())
        self._mon_dirty = True
        if L.is_torch(q2):
            return self._rt_d
        return self._host_copy(self._rt_d, self._rho_tilde)

    def freeze_upwind_state(self, grad, q2, rho, m_inf, C, m_crit, gamma=GAMMA, rho_floor=0.05):
        """(upstream, branch) copies at the current state
        (kernels/upwind.py:821-843)."""
        if self.weighted:
            raise NotImplementedError(
                "freeze_upwind_state is defined for the walk flux (weighted=False) only")
        self._walk(grad)
        d_q2, d_rho = self._state(q2, rho)
        f = self._flow(m_inf, C, m_crit, gamma, rho_floor)
        L.call("up3d_classify_branches", d_q2.data_ptr(), d_rho.data_ptr(), self._upstream_d.data_ptr(),
               self._mesh.n_tets, f, self._branch_d.data_ptr(), L.stream_ptr())
        if L.is_torch(q2):
            return self._upstream_d.clone(), self._branch_d.clone()
        return (self._host_copy(self._upstream_d, self._upstream).copy(),
                self._host_copy(self._branch_d, self._branch).copy())

    def rho_tilde_frozen(self, q2, rho, upstream, branch, m_inf, C, m_crit, gamma=GAMMA,
                         rho_floor=0.05):
        """The walk flux at a frozen (upstream, branch) assignment
        (kernels/upwind.py:845-864)."""
        t = L.torch()
        d_q2, d_rho = self._state(q2, rho)
        d_up = L.to_device(upstream, t.int64)
        d_br = L.to_device(branch, t.int8)
        f = self._flow(m_inf, C, m_crit, gamma, rho_floor)
        L.call("up3d_rho_tilde_frozen", d_q2.data_ptr(), d_rho.data_ptr(), d_up.data_ptr(), d_br.data_ptr(),
               self._mesh.n_tets, f, self._nu_d.data_ptr(), self._rt_d.data_ptr(), self._mon.data_ptr(),
               L.stream_ptr())
        self._mon_dirty = True
        if L.is_torch(q2):
            return self._rt_d
        return self._host_copy(self._rt_d, self._rho_tilde)

    def rho_tilde_frozen_sensitivities(self, q2, rho, upstream, branch, m_inf, C, m_crit,
                                       gamma=GAMMA, rho_floor=0.05):
        """(s_e, s_u) of the frozen flux (kernels/upwind.py:866-883)."""
        t = L.torch()
        d_q2, d_rho = self._state(q2, rho)
        d_up = L.to_device(upstream, t.int64)
        d_br = L.to_device(branch, t.int8)
        f = self._flow(m_inf, C, m_crit, gamma, rho_floor)
        L.call("up3d_rho_tilde_frozen_sens", d_q2.data_ptr(), d_rho.data_ptr(), d_up.data_ptr(),
               d_br.data_ptr(), self._mesh.n_tets, f, self._se_d.data_ptr(), self._su_d.data_ptr(),
               L.stream_ptr())
        if L.is_torch(q2):
            return self._se_d, self._su_d
        return self._host_copy(self._se_d, self._se), self._host_copy(self._su_d, self._su)

    def rho_tilde_sensitivities(self, grad, q2, rho, m_inf, C, m_crit, gamma=GAMMA, rho_floor=0.05):
        """(s_e, s_u, upstream) of the live walk flux at frozen selection
        (kernels/upwind.py:885-920)."""
        if self.weighted:
            raise NotImplementedError(
                "rho_tilde_sensitivities is defined for the walk flux (weighted=False) only; "
                "the weighted flux has a dense Jacobian")
        self._walk(grad)
        d_q2, d_rho = self._state(q2, rho)
        f = self._flow(m_inf, C, m_crit, gamma, rho_floor)
        L.call("up3d_rho_tilde_sens", d_q2.data_ptr(), d_rho.data_ptr(), self._upstream_d.data_ptr(),
               self._mesh.n_tets, f, self._se_d.data_ptr(), self._su_d.data_ptr(), L.stream_ptr())
        if L.is_torch(q2):
            return self._se_d, self._su_d, self._upstream_d
        return (self._host_copy(self._se_d, self._se), self._host_copy(self._su_d, self._su),
                self._host_copy(self._upstream_d, self._upstream))
