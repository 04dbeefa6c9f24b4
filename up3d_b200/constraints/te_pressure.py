"""Pressure-equality Kutta estimator on a conforming cut mesh
(pyfp3d/constraints/te_pressure.py:73-323).

Per trailing-edge node an upper and a lower control volume: the cut-mesh
tets that own a wall face and reference the TE node through its copy
("+", upper) or its original ("-", lower).  Each side's velocity is the
volume-weighted mean of its tets' P1 gradients; the station residual is
the mean over the station's TE nodes of |q_u|^2 - |q_l|^2.  Its exact
rows (dF/dphi_cut sparse, dF/dGamma dense through the copies' Gamma
dependence) feed the eliminated Newton step of the coupled solve.

Host code on the TE fans (a few tets per TE node): the gradients use the
device mesh's B, so they are the bits every other kernel uses, and only
the fan nodes' potentials cross to the host per evaluation.
"""

from __future__ import annotations

from typing import Tuple

import numpy as np
import scipy.sparse as sp

from ..mesh.wake_cut import _FaceIndex


class TEControlVolumes:
    """Wall-adjacent upper / lower TE control volumes (te_pressure.py:79-215).
    `geometry` = (B (E, 4, 3), V (E,)) of the cut mesh, host or device
    arrays; None takes it from the device mesh.  AssertionError where the
    reference raises one (wall faces not owned once, an empty side, a
    probe outside its side's volume, a far-field node in a volume)."""

    def __init__(self, mesh_cut, wc, dirichlet_nodes=None, wall_tag: str = "wall", geometry=None):
        el = np.asarray(mesh_cut.elements, dtype=np.int64)
        n_cut = len(mesh_cut.nodes)
        self.wc, self.n_te, self.n_st = wc, len(wc.te_nodes), wc.n_stations
        if self.n_te == 0:
            raise ValueError("WakeCut has no TE nodes")
        if wall_tag not in mesh_cut.boundary_faces:
            raise ValueError(f"cut mesh has no '{wall_tag}' face group")
        fidx = _FaceIndex(el)
        lo, hi = fidx.owners(np.asarray(mesh_cut.boundary_faces[wall_tag], dtype=np.int64))
        if not np.all(hi - lo == 1):
            raise AssertionError(f"{int(np.sum(hi - lo != 1))} wall faces not owned by exactly one tet")
        wall_adj = np.zeros(len(el), dtype=bool)
        wall_adj[fidx.owner[lo]] = True
        copy_of = np.full(wc.n_nodes_orig, -1, dtype=np.int64)
        copy_of[wc.master_nodes] = wc.slave_nodes
        te_copy = copy_of[wc.te_nodes]
        if np.any(te_copy < 0):
            raise AssertionError("TE node without a copy (the TE nodes must be duplicated)")
        # element stars, ascending element ids per node
        flat = el.ravel()
        order = np.argsort(flat, kind="stable")
        start = np.searchsorted(flat[order], np.arange(n_cut + 1))
        star_el = order // 4

        def fan(node):
            e = star_el[start[node]:start[node + 1]]
            return e[wall_adj[e]]

        fans_u = [fan(int(v)) for v in te_copy]
        fans_l = [fan(int(v)) for v in wc.te_nodes]
        empty = [k for k in range(self.n_te) if len(fans_u[k]) == 0 or len(fans_l[k]) == 0]
        if empty:
            raise AssertionError(f"TE nodes {empty}: empty wall-adjacent control volume on a side")
        for k in range(self.n_te):
            if wc.kutta_upper[k] not in el[fans_u[k]] or wc.kutta_lower[k] not in el[fans_l[k]]:
                raise AssertionError(f"TE node {int(wc.te_nodes[k])}: a Kutta probe outside its side's volume")
        if geometry is None:
            from ..mesh.device import get_mesh
            geometry = get_mesh(np.asarray(mesh_cut.nodes, dtype=np.float64), mesh_cut.elements).geometry()
        B_all, V_all = geometry

        def pack(fans):
            sizes = np.array([len(f) for f in fans])
            elems = np.concatenate(fans)
            seg = np.repeat(np.arange(self.n_te), sizes)
            B = _host(B_all, elems).reshape(-1, 4, 3)
            V = _host(V_all, elems)
            vsum = np.zeros(self.n_te)
            np.add.at(vsum, seg, V)
            return {"elems": elems, "seg": seg, "dofs": el[elems], "B": B, "w": V / vsum[seg], "sizes": sizes}

        self._u, self._l = pack(fans_u), pack(fans_l)
        if dirichlet_nodes is not None and len(dirichlet_nodes) > 0:
            is_dir = np.zeros(n_cut, dtype=bool)
            is_dir[np.asarray(dirichlet_nodes, dtype=np.int64)] = True
            hit = int(is_dir[self._u["dofs"]].sum() + is_dir[self._l["dofs"]].sum())
            if hit:
                raise AssertionError(f"{hit} control-volume dofs are far-field Dirichlet nodes")
        self._counts = np.bincount(wc.te_station, minlength=self.n_st).astype(np.float64)
        self._G = sp.coo_matrix((np.ones(len(wc.slave_nodes)), (wc.slave_nodes, wc.node_station)),
                                shape=(n_cut, self.n_st)).tocsr()
        self._n_cut = n_cut
        self.dofs = np.unique(np.concatenate([self._u["dofs"].ravel(), self._l["dofs"].ravel()]))

    def _phi(self, phi_cut, side):
        """Potentials at one side's fan nodes (n_fan, 4), host."""
        if hasattr(phi_cut, "is_cuda"):
            import torch
            idx = torch.as_tensor(side["dofs"].ravel(), device=phi_cut.device)
            return phi_cut[idx].cpu().numpy().reshape(-1, 4)
        return np.asarray(phi_cut, dtype=np.float64)[side["dofs"]]

    def _velocity(self, side, phi_cut):
        grad = np.einsum("ead,ea->ed", side["B"], self._phi(phi_cut, side))
        q = np.zeros((self.n_te, 3))
        np.add.at(q, side["seg"], side["w"][:, None] * grad)
        return q

    def te_velocities(self, phi_cut) -> Tuple[np.ndarray, np.ndarray]:
        """(q_upper, q_lower), (n_te, 3) each (te_pressure.py:217-228)."""
        return self._velocity(self._u, phi_cut), self._velocity(self._l, phi_cut)

    def residual_stations(self, phi_cut) -> np.ndarray:
        """F_raw per station: mean over its TE nodes of |q_u|^2 - |q_l|^2
        (te_pressure.py:230-239)."""
        qu, ql = self.te_velocities(phi_cut)
        f = np.einsum("kd,kd->k", qu, qu) - np.einsum("kd,kd->k", ql, ql)
        return np.bincount(self.wc.te_station, weights=f, minlength=self.n_st) / self._counts

    def _rows_cut(self, phi_cut, mode: str) -> sp.csr_matrix:
        """dF/dphi_cut (n_st, n_cut): "exact" 2 q_u.dq_u - 2 q_l.dq_l, or
        "frozen" (q_u + q_l).(dq_u - dq_l) (te_pressure.py:241-274)."""
        qu, ql = self.te_velocities(phi_cut)
        if mode == "exact":
            a_u, a_l = 2.0 * qu, 2.0 * ql
        elif mode == "frozen":
            a_u = a_l = qu + ql
        else:
            raise ValueError(f"unknown mode {mode!r}")
        rows, cols, vals = [], [], []
        for side, a, sign in ((self._u, a_u, 1.0), (self._l, a_l, -1.0)):
            seg = side["seg"]
            st = self.wc.te_station[seg]
            c = np.einsum("id,iad->ia", a[seg], side["B"]) * (sign * side["w"] / self._counts[st])[:, None]
            rows.append(np.repeat(st, 4))
            cols.append(side["dofs"].ravel())
            vals.append(c.ravel())
        K = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(self.n_st, self._n_cut)).tocsr()
        K.sum_duplicates()
        return K

    def gamma_jacobian(self, phi_cut, mode: str = "exact") -> np.ndarray:
        """dF/dGamma (n_st, n_st) dense (te_pressure.py:276-278)."""
        return np.asarray((self._rows_cut(phi_cut, mode) @ self._G).todense())

    def newton_rows(self, phi_cut):
        """(Kp_cut, D) exact (te_pressure.py:280-286)."""
        Kp = self._rows_cut(phi_cut, "exact")
        return Kp, np.asarray((Kp @ self._G).todense())

    def implied_targets(self, phi_cut, gamma) -> np.ndarray:
        """Gamma - M^-1 F with M the frozen-mean dF/dGamma
        (te_pressure.py:288-310)."""
        gamma = np.atleast_1d(np.asarray(gamma, dtype=np.float64))
        F = self.residual_stations(phi_cut)
        try:
            step = np.linalg.solve(self.gamma_jacobian(phi_cut, mode="frozen"), F)
        except np.linalg.LinAlgError as e:
            raise RuntimeError("frozen-mean dF/dGamma singular at this state") from e
        return gamma - step

    def fan_stats(self) -> dict:
        nu, nl = self._u["sizes"], self._l["sizes"]
        return {"n_te": self.n_te, "n_st": self.n_st, "fan_u_min": int(nu.min()),
                "fan_u_med": float(np.median(nu)), "fan_u_max": int(nu.max()), "fan_l_min": int(nl.min()),
                "fan_l_med": float(np.median(nl)), "fan_l_max": int(nl.max())}


def _host(a, idx):
    """a[idx] as a host float64 array (a host or device array)."""
    if hasattr(a, "is_cuda"):
        import torch
        return a[torch.as_tensor(idx, device=a.device)].cpu().numpy().astype(np.float64)
    return np.asarray(a, dtype=np.float64)[idx]
