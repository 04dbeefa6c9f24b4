"""Node and element renumbering of a tetrahedral mesh.

The element sweep gathers the potential and coordinates of each element's
nodes and walks to face neighbours; the row gather reads the local matrices
of each node's incident elements.  How far apart those records sit in HBM
depends on the numbering alone, so a renumbering changes the cache hit rates
and nothing else: every element keeps its local node order (its gradient
basis, face order and walk tie-breaks are unchanged), and the results of a
renumbered mesh are the original ones permuted, up to the summation order of
each node's incident elements (ascending element index).

Orderings:
  "given"   the numbering as supplied
  "morton"  nodes and elements sorted by the Morton (Z-order) key of their
            coordinates / centroids, 21 bits per axis
  "hilbert" the same with the 3-D Hilbert key (Skilling's transpose method)

The reference has no counterpart (it keeps the mesh file's numbering).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

BITS = 21
ORDERINGS = ("given", "morton", "hilbert")


def _quantise(points: np.ndarray, bits: int = BITS) -> np.ndarray:
    p = np.asarray(points, dtype=np.float64)
    lo = p.min(axis=0)
    span = p.max(axis=0) - lo
    span[span == 0] = 1.0
    q = np.floor((p - lo) / span * ((1 << bits) - 1)).astype(np.uint64)
    return np.clip(q, 0, (1 << bits) - 1)


def _spread(v: np.ndarray) -> np.ndarray:
    """Inserts two zero bits between the low 21 bits of v."""
    v = v & np.uint64(0x1FFFFF)
    v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
    return v


def morton_keys(points: np.ndarray, bits: int = BITS) -> np.ndarray:
    q = _quantise(points, bits)
    return _spread(q[:, 0]) << np.uint64(2) | _spread(q[:, 1]) << np.uint64(1) | _spread(q[:, 2])


def hilbert_keys(points: np.ndarray, bits: int = BITS) -> np.ndarray:
    return hilbert_index(_quantise(points, bits), bits)


def hilbert_index(q: np.ndarray, bits: int = BITS) -> np.ndarray:
    """3-D Hilbert index of integer coordinates q (n, 3) in [0, 2^bits):
    J. Skilling, "Programming the Hilbert curve", AIP Conf. Proc. 707
    (2004) -- axes to transposed form, then bit interleave."""
    x = np.asarray(q, dtype=np.uint64).T.copy()  # (3, n)
    n = 3
    m = np.uint64(1) << np.uint64(bits - 1)
    # inverse undo of the excess work
    q = m
    while q > 1:
        p = q - np.uint64(1)
        for i in range(n):
            hi = (x[i] & q) != 0
            # where bit set: invert low bits of x[0]; else exchange low bits of x[0] and x[i]
            x0 = x[0].copy()
            x[0] = np.where(hi, x0 ^ p, x0)
            t = np.where(hi, np.uint64(0), (x0 ^ x[i]) & p)
            x[0] = x[0] ^ t
            x[i] = x[i] ^ t
        q >>= np.uint64(1)
    # Gray encode
    for i in range(1, n):
        x[i] ^= x[i - 1]
    t = np.zeros_like(x[0])
    q = m
    while q > 1:
        t = np.where((x[n - 1] & q) != 0, t ^ (q - np.uint64(1)), t)
        q >>= np.uint64(1)
    for i in range(n):
        x[i] ^= t
    # interleave: bit b of axis i -> position 3 b + (2 - i)
    return _spread(x[0]) << np.uint64(2) | _spread(x[1]) << np.uint64(1) | _spread(x[2])


@dataclass
class Renumbered:
    """A renumbered mesh: nodes = old_nodes[node_perm], elements[e] =
    node_inv[old_elements[elem_perm[e]]] (node_perm / elem_perm map new ->
    old indices, node_inv maps old -> new)."""
    nodes: np.ndarray
    elements: np.ndarray
    node_perm: np.ndarray
    node_inv: np.ndarray
    elem_perm: np.ndarray
    elem_inv: np.ndarray
    ordering: str

    @property
    def identity(self) -> bool:
        """True for the given numbering (no permutation)."""
        return self.ordering == "given"

    def nodal(self, a):
        """An old-numbering nodal array in the new numbering."""
        return np.asarray(a)[self.node_perm]

    def nodal_back(self, a):
        """A new-numbering nodal array in the old numbering."""
        return np.asarray(a)[self.node_inv]

    def elemental(self, a):
        return np.asarray(a)[self.elem_perm]

    def elemental_back(self, a):
        return np.asarray(a)[self.elem_inv]

    def element_ids_back(self, ids):
        """New element indices (e.g. upstream elements) as old indices."""
        return self.elem_perm[np.asarray(ids)]

    def node_set(self, old_ids):
        """Old node indices (e.g. Dirichlet nodes) as new indices."""
        return np.sort(self.node_inv[np.asarray(old_ids)])


def renumber(nodes, elements, ordering: str = "morton") -> Renumbered:
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    elements = np.ascontiguousarray(elements, dtype=np.int64)
    if ordering not in ORDERINGS:
        raise ValueError(f"unknown ordering {ordering!r}; expected one of {ORDERINGS}")
    n, e = len(nodes), len(elements)
    if ordering == "given":
        node_perm = np.arange(n)
        elem_perm = np.arange(e)
    else:
        key = morton_keys if ordering == "morton" else hilbert_keys
        node_perm = np.argsort(key(nodes), kind="stable")
        elem_perm = np.argsort(key(nodes[elements].mean(axis=1)), kind="stable")
    node_inv = np.empty(n, dtype=np.int64)
    node_inv[node_perm] = np.arange(n)
    elem_inv = np.empty(e, dtype=np.int64)
    elem_inv[elem_perm] = np.arange(e)
    new_elements = node_inv[elements[elem_perm]].astype(np.int32)
    return Renumbered(nodes[node_perm], new_elements, node_perm, node_inv, elem_perm, elem_inv, ordering)
