"""The wake-cut data of a lifting mesh (pyfp3d/mesh/wake_cut.py:86-137) and
a synthetic cut of the channel mesh for tests and benchmarks.

``WakeCut`` carries what the wake constraint and the Kutta targets read:
the "+"-side copies ("slaves") of the sheet nodes appended after the
original nodes, their originals ("masters"), each copy's spanwise station,
and the trailing-edge probes.  The reference builds it from a gmsh mesh
with tagged "wake" and "wall" faces (``cut_wake``, which needs meshio and is
out of scope here); ``cut_channel_sheet`` builds the same data for a plane
sheet inside the synthetic Kuhn channel:

* the sheet is the node plane k = k_sheet downstream of the trailing-edge
  line i = i_te (all j), every sheet node duplicated;
* "+"-side elements are those of the hex layers k >= k_sheet downstream of
  the trailing edge (hexes i >= i_te); they refer to the copies, every
  other element keeps the original ids;
* one station per spanwise line j (the jump Gamma_j is constant along the
  sheet's streamwise lines, as the reference's wake lines inherit their TE
  station), station_y the line's y;
* Kutta probes one node off each TE node, upstream: (i_te - 1, j,
  k_sheet + 1) on the "+" side and (i_te - 1, j, k_sheet - 1) on the "-".
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class WakeCut:
    """Duplication map, stations and Kutta probes (attribute names of the
    reference's WakeCut)."""
    n_nodes_orig: int = 0
    master_nodes: np.ndarray = field(default_factory=lambda: np.empty(0, dtype=np.int64))
    slave_nodes: np.ndarray = field(default_factory=lambda: np.empty(0, dtype=np.int64))
    free_nodes: np.ndarray = field(default_factory=lambda: np.empty(0, dtype=np.int64))
    te_nodes: np.ndarray = field(default_factory=lambda: np.empty(0, dtype=np.int64))
    station_z: np.ndarray = field(default_factory=lambda: np.empty(0, dtype=np.float64))
    node_station: np.ndarray = field(default_factory=lambda: np.empty(0, dtype=np.int64))
    te_station: np.ndarray = field(default_factory=lambda: np.empty(0, dtype=np.int64))
    kutta_upper: np.ndarray = field(default_factory=lambda: np.empty(0, dtype=np.int64))
    kutta_lower: np.ndarray = field(default_factory=lambda: np.empty(0, dtype=np.int64))

    @property
    def n_stations(self) -> int:
        return len(self.station_z)

    def gamma_at_nodes(self, gamma_stations) -> np.ndarray:
        """(n_dup,) jump value per duplicated node from per-station Gamma."""
        return np.asarray(gamma_stations, dtype=np.float64)[self.node_station]


@dataclass
class CutMesh:
    nodes: np.ndarray        # (n_orig + n_dup, 3)
    elements: np.ndarray     # (E, 4) int32, "+"-side sheet references renumbered
    dirichlet_nodes: np.ndarray
    wc: WakeCut


def cut_channel_sheet(mesh, k_sheet: int | None = None, i_te: int | None = None,
                      single_station: bool = False) -> CutMesh:
    """A plane wake sheet cut into a Kuhn channel (module docstring)."""
    nx, ny, nz = mesh.shape
    ks = nz // 2 if k_sheet is None else int(k_sheet)
    it = nx // 2 if i_te is None else int(i_te)
    if not (1 <= ks <= nz - 1 and 1 <= it <= nx - 1):
        raise ValueError("the sheet needs interior k_sheet and i_te")
    n = mesh.n_nodes

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    ii, jj = np.meshgrid(np.arange(it, nx + 1), np.arange(ny + 1), indexing="ij")
    masters = np.sort(nid(ii, jj, ks).ravel()).astype(np.int64)
    slaves = n + np.arange(len(masters), dtype=np.int64)
    copy_of = np.full(n, -1, dtype=np.int64)
    copy_of[masters] = slaves
    # "+"-side elements: every node in the layers k >= ks and i >= it
    el = mesh.elements.astype(np.int64)
    k_of = el % (nz + 1)
    i_of = el // ((ny + 1) * (nz + 1))
    plus = np.all(k_of >= ks, axis=1) & np.all(i_of >= it, axis=1)
    el_cut = el.copy()
    sub = el_cut[plus]
    dup = copy_of[sub]
    el_cut[plus] = np.where(dup >= 0, dup, sub)
    nodes_cut = np.concatenate([mesh.nodes, mesh.nodes[masters]])
    j_of_master = (masters // (nz + 1)) % (ny + 1)
    node_station = np.zeros(len(masters), dtype=np.int64) if single_station else j_of_master
    n_st = 1 if single_station else ny + 1
    te = np.array([nid(it, j, ks) for j in range(ny + 1)], dtype=np.int64)
    te_station = np.zeros(ny + 1, dtype=np.int64) if single_station else np.arange(ny + 1, dtype=np.int64)
    station_y = np.array([mesh.nodes[te[te_station == s], 1].mean() for s in range(n_st)])
    wc = WakeCut(n_nodes_orig=n, master_nodes=masters, slave_nodes=slaves, te_nodes=te,
                 station_z=station_y, node_station=node_station, te_station=te_station,
                 kutta_upper=np.array([nid(it - 1, j, ks + 1) for j in range(ny + 1)], dtype=np.int64),
                 kutta_lower=np.array([nid(it - 1, j, ks - 1) for j in range(ny + 1)], dtype=np.int64))
    # Dirichlet nodes: the channel's, plus the copies of Dirichlet sheet nodes
    d = np.asarray(mesh.dirichlet_nodes, dtype=np.int64)
    d_dup = copy_of[d]
    dirichlet = np.sort(np.concatenate([d, d_dup[d_dup >= 0]]))
    return CutMesh(nodes_cut, el_cut.astype(np.int32), dirichlet, wc)
