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
    wake_faces_minus: np.ndarray = field(default_factory=lambda: np.empty((0, 3), dtype=np.int32))
    wake_faces_plus: np.ndarray = field(default_factory=lambda: np.empty((0, 3), dtype=np.int32))

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
    # tagged boundary triangles in cut-mesh ids ("farfield": the inflow and
    # outflow planes, the faces farfield_dirichlet reads)
    boundary_faces: dict = field(default_factory=dict)


# local node triples of a tet's four faces (face f opposite local node f)
_TET_FACES = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]], dtype=np.int64)


def _plane_faces(el_cut, el_orig, i_of_node, planes):
    """Triangles of el_cut whose three original nodes lie on one of the
    i-planes, as (n, 3) cut-mesh ids in element-major, face-minor order."""
    io = i_of_node[el_orig[:, _TET_FACES]]         # (E, 4, 3)
    on = np.zeros(io.shape[:2], dtype=bool)
    for p in planes:
        on |= np.all(io == p, axis=2)
    return el_cut[:, _TET_FACES][on].astype(np.int64)


def cut_channel_sheet(mesh, k_sheet: int | None = None, i_te: int | None = None,
                      single_station: bool = False, normal: str = "z") -> CutMesh:
    """A plane wake sheet cut into a Kuhn channel (module docstring).

    ``normal="z"`` (default): the sheet is the node plane k = k_sheet, one
    station per spanwise line j.  ``normal="y"``: the sheet is the node
    plane j = k_sheet (default ny // 2), "+"-side elements those with every
    node at j >= k_sheet downstream of the trailing edge, one station per
    line k (station coordinate z), Kutta probes (i_te - 1, j_sheet +- 1, k):
    the orientation of the reference's lifting meshes (vertical y, span z),
    under which the far-field vortex's branch cut (the ray y = y_sheet
    downstream of the vortex centre) meets the outflow plane exactly on the
    sheet."""
    if normal not in ("z", "y"):
        raise ValueError(f"normal must be 'z' or 'y', not {normal!r}")
    nx, ny, nz = mesh.shape
    n_cut_dir = nz if normal == "z" else ny
    ks = n_cut_dir // 2 if k_sheet is None else int(k_sheet)
    it = nx // 2 if i_te is None else int(i_te)
    if not (1 <= ks <= n_cut_dir - 1 and 1 <= it <= nx - 1):
        raise ValueError("the sheet needs an interior sheet plane and i_te")
    n = mesh.n_nodes

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    if normal == "z":
        ii, jj = np.meshgrid(np.arange(it, nx + 1), np.arange(ny + 1), indexing="ij")
        masters = np.sort(nid(ii, jj, ks).ravel()).astype(np.int64)
    else:
        ii, kk = np.meshgrid(np.arange(it, nx + 1), np.arange(nz + 1), indexing="ij")
        masters = np.sort(nid(ii, ks, kk).ravel()).astype(np.int64)
    slaves = n + np.arange(len(masters), dtype=np.int64)
    copy_of = np.full(n, -1, dtype=np.int64)
    copy_of[masters] = slaves
    # "+"-side elements: every node on the far side of the sheet plane and
    # downstream of the trailing edge
    el = mesh.elements.astype(np.int64)
    k_of = el % (nz + 1)
    j_of = (el // (nz + 1)) % (ny + 1)
    i_of = el // ((ny + 1) * (nz + 1))
    side = k_of if normal == "z" else j_of
    plus = np.all(side >= ks, axis=1) & np.all(i_of >= it, axis=1)
    el_cut = el.copy()
    sub = el_cut[plus]
    dup = copy_of[sub]
    el_cut[plus] = np.where(dup >= 0, dup, sub)
    nodes_cut = np.concatenate([mesh.nodes, mesh.nodes[masters]])
    if normal == "z":
        line_of_master = (masters // (nz + 1)) % (ny + 1)
        n_lines = ny + 1
        te = np.array([nid(it, j, ks) for j in range(ny + 1)], dtype=np.int64)
        up_probe = [nid(it - 1, j, ks + 1) for j in range(ny + 1)]
        lo_probe = [nid(it - 1, j, ks - 1) for j in range(ny + 1)]
        coord = 1
    else:
        line_of_master = masters % (nz + 1)
        n_lines = nz + 1
        te = np.array([nid(it, ks, k) for k in range(nz + 1)], dtype=np.int64)
        up_probe = [nid(it - 1, ks + 1, k) for k in range(nz + 1)]
        lo_probe = [nid(it - 1, ks - 1, k) for k in range(nz + 1)]
        coord = 2
    node_station = np.zeros(len(masters), dtype=np.int64) if single_station else line_of_master
    n_st = 1 if single_station else n_lines
    te_station = np.zeros(n_lines, dtype=np.int64) if single_station else np.arange(n_lines, dtype=np.int64)
    station_c = np.array([mesh.nodes[te[te_station == s], coord].mean() for s in range(n_st)])
    wc = WakeCut(n_nodes_orig=n, master_nodes=masters, slave_nodes=slaves, te_nodes=te,
                 station_z=station_c, node_station=node_station, te_station=te_station,
                 kutta_upper=np.array(up_probe, dtype=np.int64),
                 kutta_lower=np.array(lo_probe, dtype=np.int64))
    # Dirichlet nodes: the channel's, plus the copies of Dirichlet sheet nodes
    d = np.asarray(mesh.dirichlet_nodes, dtype=np.int64)
    d_dup = copy_of[d]
    dirichlet = np.sort(np.concatenate([d, d_dup[d_dup >= 0]]))
    i_of_node = np.arange(n, dtype=np.int64) // ((ny + 1) * (nz + 1))
    ff = _plane_faces(el_cut, el, i_of_node, (0, nx))
    return CutMesh(nodes_cut, el_cut.astype(np.int32), dirichlet, wc, {"farfield": ff})


def channel_vortex_center(cut: CutMesh):
    """(x, y) of the far-field vortex for a normal="y" channel cut: x of the
    trailing-edge line, y of the sheet plane, both read from boundary nodes
    (not jittered), so the vortex's branch cut meets the outflow plane
    exactly on the sheet's nodes (dy = 0 there)."""
    wc = cut.wc
    return (float(cut.nodes[wc.te_nodes[0], 0]), float(cut.nodes[wc.master_nodes[-1], 1]))


_WC_ARRAYS = ("master_nodes", "slave_nodes", "free_nodes", "te_nodes", "station_z", "node_station",
              "te_station", "kutta_upper", "kutta_lower", "wake_faces_minus", "wake_faces_plus")


def cut_arrays(mesh_cut, wc) -> dict:
    """A cut mesh and its WakeCut as flat arrays ("cut/nodes",
    "cut/elements", "cut/faces/<group>", "wc/<attribute>"), for np.savez."""
    out = {"cut/nodes": np.asarray(mesh_cut.nodes), "cut/elements": np.asarray(mesh_cut.elements),
           "wc/n_nodes_orig": np.int64(wc.n_nodes_orig)}
    for tag, faces in mesh_cut.boundary_faces.items():
        out["cut/faces/" + tag] = np.asarray(faces, dtype=np.int64)
    for k in _WC_ARRAYS:
        out["wc/" + k] = np.asarray(getattr(wc, k))
    return out


def load_cut(arrays):
    """(mesh_cut, WakeCut) from the arrays of cut_arrays (a dict or an
    NpzFile); mesh_cut carries nodes, elements and boundary_faces."""
    from types import SimpleNamespace
    keys = arrays.files if hasattr(arrays, "files") else list(arrays)
    faces = {k[len("cut/faces/"):]: np.asarray(arrays[k]) for k in keys if k.startswith("cut/faces/")}
    mc = SimpleNamespace(nodes=np.asarray(arrays["cut/nodes"]), elements=np.asarray(arrays["cut/elements"]),
                         boundary_faces=faces)
    wc = WakeCut(n_nodes_orig=int(arrays["wc/n_nodes_orig"]),
                 **{k: np.asarray(arrays["wc/" + k]) for k in _WC_ARRAYS if "wc/" + k in keys})
    return mc, wc
