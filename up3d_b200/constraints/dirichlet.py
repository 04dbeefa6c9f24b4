"""Far-field Dirichlet data of a lifting cut mesh (pyfp3d/constraints/
dirichlet.py:26-200): freestream potential plus the 2-D point-vortex
correction whose branch cut lies on the wake sheet.  Host code: it runs
once per mesh and Mach level (the Newton workspace's affine far-field
basis), on O(far-field nodes x stations) numbers.
"""

from __future__ import annotations

import numpy as np


def freestream_phi(points, alpha_deg: float = 0.0, u_inf: float = 1.0) -> np.ndarray:
    """U (x cos a + y sin a) (dirichlet.py:29-34)."""
    a = np.deg2rad(alpha_deg)
    return u_inf * (points[:, 0] * np.cos(a) + points[:, 1] * np.sin(a))


def vortex_phi_2d(points, gamma_total, center=(0.25, 0.0), lower_branch_mask=None,
                  beta: float = 1.0) -> np.ndarray:
    """-(Gamma / 2 pi) theta_w with theta_w = atan2(beta dy, dx) taken in
    [0, 2 pi): the branch cut runs along +x from the centre; points of
    `lower_branch_mask` downstream of the centre (the lower side's sheet
    nodes) take theta_w = 2 pi (dirichlet.py:37-95).  gamma_total is a
    scalar or one strength per point."""
    dx = points[:, 0] - center[0]
    dy = points[:, 1] - center[1]
    th = np.arctan2(beta * dy, dx)
    th = np.where(th < 0.0, th + 2.0 * np.pi, th)
    if lower_branch_mask is not None:
        th = np.where((dx > 0.0) & lower_branch_mask, 2.0 * np.pi, th)
    return -(gamma_total / (2.0 * np.pi)) * th


def farfield_dirichlet(mesh_cut, wc, alpha_deg: float, gamma_stations, u_inf: float = 1.0,
                       vortex_center=(0.25, 0.0), farfield_tag: str = "farfield",
                       beta: float = 1.0, spanwise_gamma: bool = False):
    """(nodes, values) on the far-field faces of the cut mesh
    (dirichlet.py:98-200): the sorted unique far-field nodes, freestream
    plus the vortex of strength mean(Gamma) -- or, with spanwise_gamma and
    several stations, of a per-node strength interpolated in z over the
    stations and held at zero from the sheet tip on."""
    ff = np.unique(np.asarray(mesh_cut.boundary_faces[farfield_tag], dtype=np.int64))
    pts = mesh_cut.nodes[ff]
    g = np.atleast_1d(np.asarray(gamma_stations, dtype=np.float64))
    lower = np.isin(ff, wc.master_nodes)
    values = freestream_phi(pts, alpha_deg, u_inf)
    if spanwise_gamma and wc.n_stations > 1:
        if np.any(g != 0.0):
            order = np.argsort(wc.station_z)
            zs, gs = wc.station_z[order], g[order]
            z_tip = float(mesh_cut.nodes[wc.master_nodes][:, 2].max())
            if z_tip > zs[-1]:
                zs = np.append(zs, z_tip)
                gs = np.append(gs, 0.0)
            strength = np.interp(pts[:, 2], zs, gs, right=0.0)
            values = values + vortex_phi_2d(pts, strength, vortex_center, lower, beta)
    else:
        g_total = float(np.mean(g))
        if g_total != 0.0:
            values = values + vortex_phi_2d(pts, g_total, vortex_center, lower, beta)
    return ff, values


class FarfieldBasis:
    """The far-field split and affine basis of a lifting case
    (NewtonWorkspace.__init__ / set_mach, solve/newton.py:224-256,
    :295-324): `dir_red` the far-field reduced rows (sorted, slaves
    dropped), `free` the rest, and per Mach level the values
    vals0_red + V_red @ Gamma, V_red found by unit-Gamma probing (the
    far-field data is linear in the station Gammas)."""

    def __init__(self, mesh_cut, wc, alpha_deg: float = 0.0, u_inf: float = 1.0,
                 vortex_center=(0.25, 0.0), spanwise_gamma: bool = False):
        self.mesh_cut, self.wc = mesh_cut, wc
        self.alpha_deg, self.u_inf = float(alpha_deg), float(u_inf)
        self.vortex_center, self.spanwise = tuple(vortex_center), bool(spanwise_gamma)
        n_red, n_st = int(wc.n_nodes_orig), wc.n_stations
        nodes, _ = farfield_dirichlet(mesh_cut, wc, self.alpha_deg, np.zeros(n_st), self.u_inf,
                                      self.vortex_center, beta=1.0, spanwise_gamma=self.spanwise)
        self.dir_cut = nodes                     # far-field nodes in cut-mesh ids
        self._keep = nodes < n_red
        self.dir_red, self._idx = np.unique(nodes[self._keep], return_index=True)
        is_dir = np.zeros(n_red, dtype=bool)
        is_dir[self.dir_red] = True
        self.is_dir = is_dir
        self.free = np.where(~is_dir)[0]

    def _reduce(self, values):
        return np.asarray(values, dtype=np.float64)[self._keep][self._idx]

    def at_mach(self, beta: float):
        """(vals0_red, V_red (n_dir, n_stations)) at Prandtl-Glauert beta."""
        n_st = self.wc.n_stations
        kw = dict(beta=beta, spanwise_gamma=self.spanwise)
        _, v0 = farfield_dirichlet(self.mesh_cut, self.wc, self.alpha_deg, np.zeros(n_st), self.u_inf,
                                   self.vortex_center, **kw)
        vals0 = self._reduce(v0)
        V = np.empty((len(self.dir_red), n_st))
        for j in range(n_st):
            e = np.zeros(n_st)
            e[j] = 1.0
            _, vj = farfield_dirichlet(self.mesh_cut, self.wc, self.alpha_deg, e, self.u_inf,
                                       self.vortex_center, **kw)
            V[:, j] = self._reduce(vj) - vals0
        return vals0, V


def kutta_row(wc, is_dir, tip_taper=None):
    """K = dF/dphi on the reduced columns (solve/newton.py:276-292): station
    row j holds +taper_j / n_j at its TE entries' upper probes and -taper_j
    / n_j at the lower ones (duplicates summed), scipy CSR (n_stations,
    n_red).  ValueError when a probe is a copy or a far-field node."""
    import scipy.sparse as sp
    n_st, n_red = wc.n_stations, len(is_dir)
    counts = np.bincount(wc.te_station, minlength=n_st).astype(np.float64)
    probes = np.concatenate([wc.kutta_upper, wc.kutta_lower]).astype(np.int64)
    if np.any(probes >= n_red) or np.any(is_dir[probes]):
        raise ValueError("Kutta probes must be free original nodes")
    w = 1.0 / counts[wc.te_station]
    rows = np.concatenate([wc.te_station, wc.te_station])
    K = sp.coo_matrix((np.concatenate([w, -w]), (rows, probes)), shape=(n_st, n_red)).tocsr()
    if tip_taper is not None and not np.all(np.asarray(tip_taper) == 1.0):
        K = (sp.diags(np.asarray(tip_taper, dtype=np.float64)) @ K).tocsr()
    K.sort_indices()
    return K
