"""The tiled assembly's plan, built on the host (no device): a CPU
emulation of the tile kernel's summation (each tile's outputs from its
elements' local values in the plan's order, written whole when the tile
holds every contributor, else as partials that the combine pass adds in
tile order) reproduces a direct scatter of the same local values into R
and the P1 Jacobian, every output written exactly once; the renumbering is
a permutation that keeps each tile inside one connected component; the
local connectivity and the internal face-neighbour table match the
mesh's."""

import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

PAIRS = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
ARRAYS = {"perm": np.int32, "iperm": np.int32, "eoff": np.int32, "noff": np.int32, "uoff": np.int32,
          "tnode": np.int32, "lconn": np.uint16, "nent_off": np.int32, "nent": np.uint16, "ndst": np.int32,
          "uent_off": np.int32, "uent": np.uint16, "udst": np.int32, "cn_off": np.int32, "cn_idx": np.int32,
          "cn_dst": np.int32, "ce_off": np.int32, "ce_idx": np.int32, "ce_dst": np.int32, "fnbr": np.int32}


def _pattern(elements, n):
    r = np.repeat(elements, 4, axis=1).ravel()
    c = np.tile(elements, (1, 4)).ravel()
    P = sp.csr_matrix((np.ones(len(r)), (r, c)), shape=(n, n))
    P.sum_duplicates()
    P.sort_indices()
    return P.indptr.astype(np.int32), P.indices.astype(np.int32)


def _plan(nodes, elements, T, stretch=1):
    from oracle import oracle as O
    from up3d_b200 import _lib as L
    el = np.ascontiguousarray(elements, dtype=np.int32)
    fn = np.ascontiguousarray(O.UpwindOperator(nodes, elements).face_neighbors, dtype=np.int32)
    cen = np.ascontiguousarray(nodes[el].mean(axis=1))
    indptr, indices = _pattern(el, len(nodes))
    h = ctypes.c_void_p()
    L.call("up3d_tile_plan_host_create", el.ctypes.data, fn.ctypes.data, cen.ctypes.data, len(nodes), len(el),
           indptr.ctypes.data, indices.ctypes.data, T, stretch, ctypes.byref(h))
    try:
        info = L.TileInfo()
        L.call("up3d_tile_plan_host_info", h, ctypes.byref(info))
        out = {"info": info.as_dict(), "indptr": indptr, "indices": indices, "fn_user": fn}
        for name, dt in ARRAYS.items():
            nb = ctypes.c_int64()
            L.call("up3d_tile_plan_host_array", h, name.encode(), None, ctypes.byref(nb))
            a = np.empty(nb.value // np.dtype(dt).itemsize, dtype=dt)
            L.call("up3d_tile_plan_host_array", h, name.encode(), a.ctypes.data, ctypes.byref(nb))
            out[name] = a
    finally:
        L.lib().up3d_tile_plan_host_destroy(h)
    for k in ("lconn", "fnbr"):
        out[k] = out[k].reshape(-1, 4)
    for k in ("ndst", "udst", "cn_dst", "ce_dst"):
        out[k] = out[k].reshape(-1, 2)
    return out


def _meshes():
    from up3d_b200.mesh.kuhn import bump_channel
    one = bump_channel(14, 6, 5, amplitude=0.08, seed=1)
    a = bump_channel(9, 4, 3, amplitude=0.05, seed=2)
    b = bump_channel(11, 5, 4, amplitude=0.03, seed=3)
    # two disconnected cases in one mesh, plus an isolated node
    nodes = np.vstack([a.nodes, b.nodes, [[9.0, 9.0, 9.0]]])
    elements = np.vstack([a.elements, b.elements + len(a.nodes)]).astype(np.int32)
    return [("channel", one.nodes, one.elements, [len(one.elements)]),
            ("union", nodes, elements, [len(a.elements), len(b.elements)])]


@pytest.mark.parametrize("T,stretch", [(128, 1), (256, 1), (256, 4)])
@pytest.mark.parametrize("case", [0, 1])
def test_plan_reproduces_a_direct_scatter(case, T, stretch):
    name, nodes, elements, comp_sizes = _meshes()[case]
    P = _plan(nodes, elements, T, stretch)
    assert P["info"]["tile_stretch"] == stretch
    E, N = len(elements), len(nodes)
    indptr, indices = P["indptr"], P["indices"]
    Z = len(indices)
    perm, iperm, eoff = P["perm"], P["iperm"], P["eoff"]
    # renumbering and tiles
    assert np.array_equal(np.sort(perm), np.arange(E)) and np.array_equal(iperm[perm], np.arange(E))
    sizes = np.diff(eoff)
    assert sizes.min() > 0 and sizes.max() <= T and eoff[-1] == E
    comp = np.repeat(np.arange(len(comp_sizes)), comp_sizes)
    for t in range(len(sizes)):
        assert len(np.unique(comp[perm[eoff[t]:eoff[t + 1]]])) == 1
        assert np.all(np.diff(perm[eoff[t]:eoff[t + 1]]) > 0)  # ascending user id inside a tile
    # local connectivity and the internal neighbour table
    for t in range(len(sizes)):
        tn = P["tnode"][P["noff"][t]:P["noff"][t + 1]]
        assert np.array_equal(tn[P["lconn"][eoff[t]:eoff[t + 1]]], elements[perm[eoff[t]:eoff[t + 1]]])
    fu = P["fn_user"][perm]
    assert np.array_equal(P["fnbr"], np.where(fu >= 0, iperm[np.maximum(fu, 0)], -1))

    # local values in user order; the direct scatter
    rng = np.random.default_rng(7)
    loc = rng.standard_normal((E, 14))
    R_ref = np.zeros(N)
    J_ref = sp.csr_matrix((N, N))
    rows, cols, vals = [], [], []
    for i in range(4):
        np.add.at(R_ref, elements[:, i], loc[:, 2 * i])
        rows.append(elements[:, i]); cols.append(elements[:, i]); vals.append(loc[:, 2 * i + 1])
    for k, (i, j) in enumerate(PAIRS):
        rows += [elements[:, i], elements[:, j]]
        cols += [elements[:, j], elements[:, i]]
        vals += [loc[:, 8 + k], loc[:, 8 + k]]
    J_ref = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    J_ref.sum_duplicates()
    J_ref.sort_indices()

    # the emulated tile kernel + combine
    R = np.full(N, np.nan)
    J = np.full(Z, np.nan)
    written_R = np.zeros(N, dtype=int)
    written_J = np.zeros(Z, dtype=int)
    part = np.full(P["info"]["n_partials"], np.nan)
    for t in range(len(sizes)):
        lv = loc[perm[eoff[t]:eoff[t + 1]]]
        for p in range(P["noff"][t], P["noff"][t + 1]):
            codes = P["nent"][P["nent_off"][p]:P["nent_off"][p + 1]].astype(int)
            assert np.all(np.diff(codes >> 2) > 0)  # ascending local element
            rs = ds = 0.0
            for c in codes:
                rs += lv[c >> 2, 2 * (c & 3)]
                ds += lv[c >> 2, 2 * (c & 3) + 1]
            dx, dy = P["ndst"][p]
            if dx >= 0:
                R[dx] = rs
                J[dy] = ds
                written_R[dx] += 1
                written_J[dy] += 1
            else:
                q = -1 - dx
                part[q], part[q + 1] = rs, ds
        for p in range(P["uoff"][t], P["uoff"][t + 1]):
            codes = P["uent"][P["uent_off"][p]:P["uent_off"][p + 1]].astype(int)
            v = 0.0
            for c in codes:
                v += lv[c >> 3, 8 + (c & 7)]
            dx, dy = P["udst"][p]
            if dx >= 0:
                J[dx] = J[dy] = v
                written_J[dx] += 1
                written_J[dy] += 1
            else:
                part[-1 - dx] = v
    assert not np.isnan(part).any()
    for k in range(len(P["cn_dst"])):
        qs = P["cn_idx"][P["cn_off"][k]:P["cn_off"][k + 1]]
        n, d = P["cn_dst"][k]
        R[n] = sum(part[q] for q in qs) if len(qs) else 0.0
        written_R[n] += 1
        if d >= 0:
            J[d] = sum(part[q + 1] for q in qs)
            written_J[d] += 1
    for k in range(len(P["ce_dst"])):
        qs = P["ce_idx"][P["ce_off"][k]:P["ce_off"][k + 1]]
        s, z = P["ce_dst"][k]
        J[s] = J[z] = sum(part[q] for q in qs)
        written_J[s] += 1
        written_J[z] += 1
    assert np.all(written_R == 1) and np.all(written_J == 1)
    assert np.abs(R - R_ref).max() <= 1e-13 * np.abs(R_ref).max()
    assert np.array_equal(J_ref.indptr, indptr) and np.array_equal(J_ref.indices, indices)
    assert np.abs(J - J_ref.data).max() <= 1e-13 * np.abs(J_ref.data).max()
    if name == "union":
        assert R[N - 1] == 0.0  # the isolated node: R = 0, no row


def test_plan_rejects_a_bad_tile_size():
    from up3d_b200 import _lib as L
    _, nodes, elements, _ = _meshes()[0]
    with pytest.raises(ValueError, match="tile_elems"):
        _plan(nodes, elements, 100)
    assert L.lib() is not None
