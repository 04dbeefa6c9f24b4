"""Cut-element census and extended-DOF numbering of the level-set wake,
with the reference's interface (pyfp3d/wake/cut_elements.py:77-333).

Rules (the reference's, restated):

* node side: the sign of the level-set offset s, with nodes within
  eps_rel x (shortest incident edge) of the sheet, and every TE node, moved
  to the "+" side, so no node sits on the sheet;
* TE nodes: |s| and |d| both below te_tol_rel x (shortest incident edge),
  optionally only among the given wall nodes;
* cut elements: elements whose nodes change side where the s = 0 crossing
  of some edge lies on the sheet: downstream of the TE (d > 0) and within
  its span (0 <= q <= span_length + outboard_fringe; the inboard test can be
  replaced by a caller's clip of the crossing points; an infinite fringe
  drops the outboard test); elements crossing downstream but off the span
  are reported as beyond_tip_elems;
* the below-TE fan (an element with a TE node whose other nodes are all
  "-") is not cut: te_lower_elems;
* one aux DOF per distinct node of the cut elements, numbered n_main + k
  in ascending node order; a cut element's upper copy takes the main DOF at
  "+" nodes and the aux DOF at "-" nodes, the lower copy the complement.

Host numpy, once per mesh and level set (not a hot path).
"""

from __future__ import annotations

from typing import Dict, Optional

import numpy as np

TET_EDGES = np.array([(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)], dtype=np.int64)


def shortest_incident_edge(nodes: np.ndarray, elements: np.ndarray) -> np.ndarray:
    """(n_nodes,) length of each node's shortest element edge (inf if the
    node is in no element)."""
    el = np.asarray(elements, dtype=np.int64)
    a = el[:, TET_EDGES[:, 0]].ravel()
    b = el[:, TET_EDGES[:, 1]].ravel()
    length = np.linalg.norm(nodes[a] - nodes[b], axis=1)
    h = np.full(len(nodes), np.inf)
    np.minimum.at(h, a, length)
    np.minimum.at(h, b, length)
    return h


class CutElementMap:
    """Side marking, cut census and extended-DOF numbering (module
    docstring).  Attributes as the reference's: s_raw, d, q, s, node_side,
    shifted_nodes, te_nodes, cut_elems, beyond_tip_elems, te_lower_elems,
    n_main, n_ext_dofs, n_total_dofs, ext_dof_of_node, dofs_upper,
    dofs_lower, span_length, outboard_fringe, wall_nodes."""

    def __init__(self, nodes, elements, levelset, wall_nodes=None, eps_rel: float = 1e-6,
                 te_tol_rel: float = 1e-3, inboard_clip=None, outboard_fringe: float = 0.0):
        nodes = np.asarray(nodes, dtype=np.float64)
        el = np.asarray(elements, dtype=np.int64)
        n = len(nodes)
        self.n_main = n
        self.wall_nodes = None if wall_nodes is None else np.asarray(wall_nodes, dtype=np.int64)
        if outboard_fringe < 0.0:
            raise ValueError("outboard_fringe must be >= 0")
        self.outboard_fringe = float(outboard_fringe)
        self.span_length = levelset.span_length
        s_raw, d, q = levelset.evaluate(nodes)
        self.s_raw, self.d, self.q = s_raw, d, q
        h = shortest_incident_edge(nodes, el)

        te = (np.abs(s_raw) < te_tol_rel * h) & (np.abs(d) < te_tol_rel * h)
        if self.wall_nodes is not None:
            wall = np.zeros(n, dtype=bool)
            wall[self.wall_nodes] = True
            te &= wall
        self.te_nodes = np.flatnonzero(te)

        eps = eps_rel * h
        moved = (np.abs(s_raw) < eps) | te
        s = s_raw.copy()
        s[moved] = eps[moved]
        self.s = s
        self.shifted_nodes = np.flatnonzero(moved)
        self.node_side = np.where(s > 0.0, 1, -1).astype(np.int8)

        side = self.node_side[el]
        cand = np.flatnonzero(side.min(axis=1) != side.max(axis=1))
        ea, eb = TET_EDGES[:, 0], TET_EDGES[:, 1]
        sc, dc, qc = s[el[cand]], d[el[cand]], q[el[cand]]
        sa, sb = sc[:, ea], sc[:, eb]
        crosses = sa * sb < 0.0
        with np.errstate(divide="ignore", invalid="ignore"):
            f = np.where(crosses, sa / (sa - sb), 0.0)
        d_x = dc[:, ea] + f * (dc[:, eb] - dc[:, ea])
        q_x = qc[:, ea] + f * (qc[:, eb] - qc[:, ea])
        downstream = crosses & (d_x > 0.0)
        if np.isinf(self.outboard_fringe):
            on_sheet = downstream
        else:
            on_sheet = downstream & (q_x <= self.span_length + self.outboard_fringe)
        if inboard_clip is None:
            on_sheet &= q_x >= 0.0
        else:
            xyz = nodes[el[cand]]
            pa, pb = xyz[:, ea, :], xyz[:, eb, :]
            inside = np.asarray(inboard_clip(pa + f[:, :, None] * (pb - pa)), dtype=bool)
            if inside.shape != crosses.shape:
                raise ValueError(f"inboard_clip returned {inside.shape}, expected {crosses.shape}")
            on_sheet &= inside
        hit = on_sheet.any(axis=1)
        cut = cand[hit]
        self.beyond_tip_elems = cand[downstream.any(axis=1) & ~hit]

        is_te = np.zeros(n, dtype=bool)
        is_te[self.te_nodes] = True
        te_e = is_te[el]
        fan = te_e.any(axis=1) & np.all(te_e | (side == -1), axis=1)
        self.te_lower_elems = np.flatnonzero(fan)
        self.cut_elems = cut[~fan[cut]]

        cut_nodes = np.unique(el[self.cut_elems])
        self.n_ext_dofs = len(cut_nodes)
        self.n_total_dofs = n + self.n_ext_dofs
        self.ext_dof_of_node = np.full(n, -1, dtype=np.int64)
        self.ext_dof_of_node[cut_nodes] = n + np.arange(self.n_ext_dofs, dtype=np.int64)
        if len(self.te_nodes) and self.n_ext_dofs and not (self.ext_dof_of_node[self.te_nodes] >= 0).all():
            raise ValueError("a TE node is in no cut element (the sheet does not reach the TE)")

        conn = el[self.cut_elems]
        aux = self.ext_dof_of_node[conn]
        plus = self.node_side[conn] == 1
        self.dofs_upper = np.where(plus, conn, aux)
        self.dofs_lower = np.where(plus, aux, conn)

    def summary(self) -> Dict[str, int]:
        return {"n_main": int(self.n_main), "n_ext_dofs": int(self.n_ext_dofs),
                "n_cut_elems": int(len(self.cut_elems)), "n_te_nodes": int(len(self.te_nodes)),
                "n_te_lower_elems": int(len(self.te_lower_elems)),
                "n_beyond_tip_elems": int(len(self.beyond_tip_elems)),
                "n_shifted_nodes": int(len(self.shifted_nodes)),
                "n_side_plus": int(np.sum(self.node_side == 1)), "n_side_minus": int(np.sum(self.node_side == -1))}
