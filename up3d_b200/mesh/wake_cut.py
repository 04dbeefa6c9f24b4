"""The wake cut of a lifting mesh (pyfp3d/mesh/wake_cut.py:59-594) and a
synthetic cut of the channel mesh for tests and benchmarks.

``WakeCut`` carries what the wake constraint and the Kutta targets read:
the "+"-side copies ("slaves") of the sheet nodes appended after the
original nodes, their originals ("masters"), each copy's spanwise station,
and the trailing-edge probes.  ``cut_wake`` builds it from a mesh with a
tagged interior "wake" face group and a "wall" group (as read by
``mesh.reader.read_mesh``); ``assert_wake_topology`` checks the result.
``cut_channel_sheet`` builds the same data for a plane sheet inside the
synthetic Kuhn channel:

* the sheet is the node plane k = k_sheet (or j = j_sheet) downstream of
  the trailing-edge line i = i_te, every sheet node duplicated;
* "+"-side elements are those of the hex layers on the far side of the
  sheet downstream of the trailing edge; they refer to the copies, every
  other element keeps the original ids;
* one station per spanwise line (the jump Gamma_j is constant along the
  sheet's streamwise lines, as the reference's wake lines inherit their TE
  station);
* Kutta probes one node off each TE node, upstream, one on each side.
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


# ------------------------------------------------------------------ cut_wake

def _row_keys(rows) -> np.ndarray:
    """Order-independent keys of node tuples (each row sorted, viewed as
    one opaque record): equal keys <=> same node set."""
    a = np.ascontiguousarray(np.sort(np.asarray(rows, dtype=np.int64), axis=1))
    return a.view(np.dtype((np.void, 8 * a.shape[1]))).ravel()


class _FaceIndex:
    """Every tet face (4 per tet, face f opposite local node f) sorted by
    key, to find the owners of given triangles."""

    def __init__(self, elements64):
        faces = elements64[:, _TET_FACES].reshape(-1, 3)
        keys = _row_keys(faces)
        self.order = np.argsort(keys, kind="stable")
        self.keys = keys[self.order]
        self.owner = (np.arange(len(faces)) // 4)[self.order]

    def owners(self, tris):
        """(lo, hi) ranges into self.owner per triangle."""
        k = _row_keys(tris)
        return np.searchsorted(self.keys, k, side="left"), np.searchsorted(self.keys, k, side="right")


def _sheet_free_nodes(boundary_faces, wake_faces, wake_tag):
    """Nodes of the sheet's interior free edges (wake_cut.py:146-177): sheet
    edges used by one wake face that are not edges of any other boundary
    triangle."""
    def edges(t):
        t = np.asarray(t, dtype=np.int64)
        return np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    k, c = np.unique(_row_keys(edges(wake_faces)), return_counts=True)
    rim = k[c == 1]
    if len(rim) == 0:
        return np.empty(0, dtype=np.int64)
    other = [edges(t) for tag, t in boundary_faces.items() if tag != wake_tag and len(t)]
    if other:
        rim = rim[~np.isin(rim, np.unique(_row_keys(np.concatenate(other))))]
    if len(rim) == 0:
        return np.empty(0, dtype=np.int64)
    return np.unique(np.frombuffer(rim.tobytes(), dtype=np.int64))


def cut_wake(mesh, wake_tag: str = "wake", wall_tag: str = "wall", upper_hint=(0.0, 1.0, 0.0)):
    """Duplicate the wake-sheet nodes and attach the "+"-side elements and
    boundary faces to the copies (wake_cut.py:225-441).  Returns (mesh_cut,
    wc): a new ``reader.Mesh`` whose boundary groups have `wake_tag`
    replaced by "wake_minus" / "wake_plus", and the ``WakeCut``.

    The "+" side of each wake face is the owner whose centroid lies further
    along upper_hint.  A duplicated node's element star is split into the
    components connected through faces that contain the node and are not
    wake faces -- exactly two, one of them holding the "+" owners of every
    wake face at the node -- computed for all nodes at once as the
    connected components of the (node, element) incidences.  Nodes on the
    sheet's interior free edges stay single-valued; TE nodes (sheet and
    wall) are duplicated.  Stations group the TE nodes by (x, y) rounded to
    1e-6 of the bounding box, numbered in lexicographic key order; every
    copy takes the station nearest in z.  Kutta probes: per TE node, the
    nearest wall neighbour (sharing a wall triangle, not on the sheet) on
    each side of upper_hint, first among neighbours in the TE node's z
    plane, else among all (ties by the smaller node id).
    AssertionError where the reference raises one (non-conforming sheet,
    ambiguous sides, a star not split in two, missing probes)."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    from .reader import Mesh
    if wake_tag not in mesh.boundary_faces:
        raise ValueError(f"mesh has no '{wake_tag}' face group")
    if wall_tag not in mesh.boundary_faces:
        raise ValueError(f"mesh has no '{wall_tag}' face group")
    nodes = np.asarray(mesh.nodes, dtype=np.float64)
    el = np.asarray(mesh.elements, dtype=np.int64)
    n = len(nodes)
    hint = np.asarray(upper_hint, dtype=np.float64)
    hint = hint / np.linalg.norm(hint)
    wake = np.asarray(mesh.boundary_faces[wake_tag], dtype=np.int64)
    fidx = _FaceIndex(el)
    lo, hi = fidx.owners(wake)
    if np.any(hi - lo != 2):
        raise AssertionError(f"{int(np.sum(hi - lo != 2))} wake face(s) not shared by exactly two tets "
                             "(sheet does not conform to the volume mesh)")
    own = np.stack([fidx.owner[lo], fidx.owner[lo + 1]], axis=1)
    cen = nodes[el].mean(axis=1)
    fc = nodes[wake].mean(axis=1)
    side = np.einsum("fkx,x->fk", cen[own] - fc[:, None, :], hint)
    if np.any(side[:, 0] == side[:, 1]):
        raise AssertionError(f"wake face {int(np.argmax(side[:, 0] == side[:, 1]))}: cannot classify sides "
                             f"along upper_hint {tuple(hint)}")
    plus_owner = np.where(side[:, 0] > side[:, 1], own[:, 0], own[:, 1])

    wake_nodes = np.unique(wake)
    wall = np.asarray(mesh.boundary_faces[wall_tag], dtype=np.int64)
    wall_nodes = np.unique(wall)
    free = _sheet_free_nodes(mesh.boundary_faces, wake, wake_tag)
    is_wall = np.zeros(n, dtype=bool)
    is_wall[wall_nodes] = True
    is_free = np.zeros(n, dtype=bool)
    is_free[free] = True
    te = wake_nodes[is_wall[wake_nodes] & ~is_free[wake_nodes]]
    dup = wake_nodes[~is_free[wake_nodes]]
    if len(te) == 0:
        raise AssertionError("wake sheet does not touch the wall (no TE nodes)")

    # stations
    zext = float(np.ptp(nodes[:, 2]))
    z_tol = 1e-9 * zext if zext > 0 else 1e-12
    bbox = float(np.max(np.ptp(nodes, axis=0)))
    xy = np.round(nodes[te, :2] / (1e-6 * bbox)).astype(np.int64)
    _, te_station = np.unique(xy, axis=0, return_inverse=True)
    te_station = te_station.astype(np.int64).ravel()
    n_st = int(te_station.max()) + 1
    station_z = np.array([nodes[te[te_station == j], 2].mean() for j in range(n_st)])
    if n_st == 1:
        node_station = np.zeros(len(dup), dtype=np.int64)
    else:
        order = np.argsort(station_z)
        sz = station_z[order]
        z = nodes[dup, 2]
        right = np.clip(np.searchsorted(sz, z), 0, n_st - 1)
        left = np.clip(right - 1, 0, n_st - 1)
        node_station = order[np.where(np.abs(z - sz[left]) < np.abs(z - sz[right]), left, right)]

    # (node, element) incidences of the duplicated nodes and their
    # connections across non-wake faces that contain the node
    dup_index = np.full(n, -1, dtype=np.int64)
    dup_index[dup] = np.arange(len(dup))
    inc_e, inc_l = np.nonzero(dup_index[el] >= 0)                 # element, local slot
    inc_d = dup_index[el[inc_e, inc_l]]
    key = inc_d * len(el) + inc_e                                 # unique per incidence
    korder = np.argsort(key)
    key_sorted = key[korder]

    def inc_id(d, e):
        k = d * len(el) + e
        pos = np.searchsorted(key_sorted, k)
        return korder[pos]

    # interior faces: consecutive equal keys in the face index
    same = fidx.keys[1:] == fidx.keys[:-1]
    f_lo = np.nonzero(same)[0]
    e1, e2 = fidx.owner[f_lo], fidx.owner[f_lo + 1]
    face_local = fidx.order[f_lo] % 4                             # face of e1 (opposite this slot)
    tri1 = el[e1[:, None], np.array(_TET_FACES)[face_local]]      # the face's nodes
    wake_keys = np.sort(_row_keys(wake))
    fk = fidx.keys[f_lo]
    pos = np.clip(np.searchsorted(wake_keys, fk), 0, max(len(wake_keys) - 1, 0))
    not_wake = ~((len(wake_keys) > 0) & (wake_keys[pos] == fk)) if len(wake_keys) else np.ones(len(fk), bool)
    rows, cols = [], []
    for j in range(3):
        d = dup_index[tri1[:, j]]
        m = not_wake & (d >= 0)
        rows.append(inc_id(d[m], e1[m]))
        cols.append(inc_id(d[m], e2[m]))
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    n_inc = len(inc_d)
    graph = coo_matrix((np.ones(len(rows)), (rows, cols)), shape=(n_inc, n_inc))
    _, label = connected_components(graph, directed=False)
    # two components per duplicated node
    pair = np.unique(np.stack([inc_d, label], axis=1), axis=0)
    n_comp = np.bincount(pair[:, 0], minlength=len(dup))
    if np.any(n_comp != 2):
        bad = int(dup[np.argmax(n_comp != 2)])
        raise AssertionError(f"wake node {bad}: element star splits into {int(n_comp[dup_index[bad]])} "
                             "components (expected 2)")
    # the "+" component of each node: the label of every (node, plus owner)
    fd = dup_index[wake]                                          # (n_wake, 3)
    m = fd >= 0
    d_of = fd[m]
    lab = label[inc_id(d_of, np.broadcast_to(plus_owner[:, None], fd.shape)[m])]
    plus_label = np.full(len(dup), -1, dtype=np.int64)
    plus_label[d_of] = lab
    if np.any(plus_label[d_of] != lab):
        bad = int(dup[d_of[np.argmax(plus_label[d_of] != lab)]])
        raise AssertionError(f"wake node {bad}: inconsistent +/- side classification across its wake faces")
    on_plus = label == plus_label[inc_d]
    slaves = n + np.arange(len(dup), dtype=np.int64)
    el_cut = el.copy()
    el_cut[inc_e[on_plus], inc_l[on_plus]] = slaves[inc_d[on_plus]]

    # boundary faces owned by a "+"-side element take the copies
    faces_cut = {}
    for tag, tris in mesh.boundary_faces.items():
        if tag == wake_tag:
            continue
        t = np.asarray(tris, dtype=np.int64).copy()
        touched = np.nonzero((dup_index[t] >= 0).any(axis=1))[0]
        if len(touched):
            blo, bhi = fidx.owners(t[touched])
            if np.any(bhi - blo != 1):
                raise AssertionError(f"boundary face in '{tag}' owned by {int((bhi - blo)[bhi - blo != 1][0])} tets")
            e = fidx.owner[blo]
            for j in range(3):
                d = dup_index[t[touched, j]]
                ok = d >= 0
                flip = np.zeros(len(touched), dtype=bool)
                flip[ok] = on_plus[inc_id(d[ok], e[ok])]
                t[touched[flip], j] = slaves[d[flip]]
        faces_cut[tag] = np.ascontiguousarray(t, dtype=np.int32)
    wake_plus = wake.copy()
    wake_plus[m] = slaves[fd[m]]
    faces_cut["wake_minus"] = np.ascontiguousarray(wake, dtype=np.int32)
    faces_cut["wake_plus"] = np.ascontiguousarray(wake_plus, dtype=np.int32)

    mc = Mesh()
    mc.nodes = np.vstack([nodes, nodes[dup]])
    mc.elements = np.ascontiguousarray(el_cut, dtype=np.int32)
    mc.boundary_faces = faces_cut
    mc.element_tags = np.asarray(mesh.element_tags).copy()
    mc.tag_names = list(mesh.tag_names)
    mc.name = f"{mesh.name}_cut"
    mc.validate()
    wc = WakeCut(n_nodes_orig=n, master_nodes=dup, slave_nodes=slaves, free_nodes=free, te_nodes=te,
                 station_z=station_z, node_station=node_station, te_station=te_station,
                 wake_faces_minus=faces_cut["wake_minus"], wake_faces_plus=faces_cut["wake_plus"])
    wc.kutta_upper, wc.kutta_lower = _kutta_probes(nodes, wall, wake_nodes, te, hint, z_tol)
    assert_wake_topology(mc, wc)
    return mc, wc


def _kutta_probes(nodes, wall, wake_nodes, te, hint, z_tol):
    """Per TE node the nearest wall neighbour on each side of hint
    (wake_cut.py:444-506)."""
    n = len(nodes)
    excluded = np.zeros(n, dtype=bool)
    excluded[wake_nodes] = True
    excluded[te] = True
    te_pos = np.full(n, -1, dtype=np.int64)
    te_pos[te] = np.arange(len(te))
    # (TE node, wall neighbour) pairs from the wall triangles
    a = np.concatenate([wall[:, [0, 1]], wall[:, [1, 0]], wall[:, [0, 2]], wall[:, [2, 0]],
                        wall[:, [1, 2]], wall[:, [2, 1]]])
    a = a[(te_pos[a[:, 0]] >= 0) & ~excluded[a[:, 1]]]
    a = np.unique(a, axis=0)
    t, nb = a[:, 0], a[:, 1]
    off = nodes[nb] - nodes[t]
    side = off @ hint
    dist = np.linalg.norm(off, axis=1)
    plane = np.abs(nodes[nb, 2] - nodes[t, 2]) <= 10 * z_tol + 1e-12
    upper = np.full(len(te), -1, dtype=np.int64)
    lower = np.full(len(te), -1, dtype=np.int64)

    def pick(mask, out):
        idx = np.nonzero(mask)[0]
        # nearest first, then the smaller node id
        idx = idx[np.lexsort((nb[idx], dist[idx], te_pos[t[idx]]))]
        first = np.unique(te_pos[t[idx]], return_index=True)
        sel = np.full(len(te), -1, dtype=np.int64)
        sel[first[0]] = nb[idx[first[1]]]
        return np.where(out < 0, sel, out)

    for restrict in (True, False):
        need = (upper < 0) | (lower < 0)
        if not need.any():
            break
        keep = need[te_pos[t]] & (plane if restrict else True)
        u = pick(keep & (side > 0), np.full(len(te), -1, dtype=np.int64))
        l_ = pick(keep & (side < 0), np.full(len(te), -1, dtype=np.int64))
        both = need & (u >= 0) & (l_ >= 0) if restrict else need
        upper = np.where(both, u, upper)
        lower = np.where(both, l_, lower)
    if np.any(upper < 0) or np.any(lower < 0):
        missing = te[(upper < 0) | (lower < 0)].tolist()
        raise AssertionError(f"TE nodes {missing}: no wall node one edge off the TE on both sides (Kutta probes)")
    return upper, lower


def assert_wake_topology(mesh_cut, wc) -> None:
    """The cut's invariants (wake_cut.py:509-594): each wake_minus /
    wake_plus face owned by one tet; TE nodes duplicated; every copy used;
    copies = sheet nodes minus free-edge nodes; no element holds a master
    and its own copy; every boundary face owned by one tet."""
    el = np.asarray(mesh_cut.elements, dtype=np.int64)
    fidx = _FaceIndex(el)
    for tag in ("wake_minus", "wake_plus"):
        lo, hi = fidx.owners(mesh_cut.boundary_faces[tag])
        assert np.all(hi - lo == 1), f"{tag}: {int(np.sum(hi - lo != 1))} face(s) not owned by exactly one tet"
    assert np.isin(wc.te_nodes, wc.master_nodes).all(), "TE node(s) missing from the duplication map"
    used = np.zeros(len(mesh_cut.nodes), dtype=bool)
    used[el.ravel()] = True
    assert used[wc.slave_nodes].all(), f"{int((~used[wc.slave_nodes]).sum())} orphan duplicated node(s)"
    assert len(wc.slave_nodes) == len(np.unique(wc.wake_faces_minus)) - len(wc.free_nodes), \
        "duplicated-node count differs from sheet nodes minus free-edge nodes"
    master_of = np.full(len(mesh_cut.nodes), -1, dtype=np.int64)
    master_of[wc.slave_nodes] = wc.master_nodes
    m = master_of[el]                                             # the master of each copy slot
    clash = (m[:, :, None] >= 0) & (m[:, :, None] == el[:, None, :])
    assert not clash.any(), f"element {int(np.argmax(clash.any(axis=(1, 2))))} references a master and its own copy"
    for tag, tris in mesh_cut.boundary_faces.items():
        lo, hi = fidx.owners(tris)
        assert np.all(hi - lo == 1), f"boundary group '{tag}': {int(np.sum(hi - lo != 1))} face(s) not owned by one tet"
