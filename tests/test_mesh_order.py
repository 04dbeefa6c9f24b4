"""Mesh renumbering (space-filling-curve orderings): the keys, the
permutations and what a renumbered mesh keeps."""

import numpy as np
import pytest


def test_hilbert_index_is_a_unit_step_curve():
    from up3d_b200.mesh.order import hilbert_index
    g = np.stack(np.meshgrid(np.arange(8), np.arange(8), np.arange(8), indexing="ij"), -1).reshape(-1, 3)
    k = hilbert_index(g, bits=3)
    assert np.array_equal(np.sort(k), np.arange(512, dtype=np.uint64))
    path = g[np.argsort(k)]
    steps = np.abs(np.diff(path, axis=0)).sum(axis=1)
    assert np.all(steps == 1)


def test_morton_keys_interleave_bits():
    from up3d_b200.mesh.order import _spread, morton_keys
    assert int(_spread(np.array([0b101], dtype=np.uint64))[0]) == 0b1000001
    pts = np.array([[0, 0, 0], [0, 0, 1], [0, 1, 0], [1, 0, 0], [1, 1, 1]], dtype=np.float64)
    k = morton_keys(pts)
    assert list(np.argsort(k)) == [0, 1, 2, 3, 4]
    assert k[1] < k[2] < k[3]


@pytest.mark.parametrize("ordering", ["given", "morton", "hilbert"])
def test_renumber_keeps_the_mesh(ordering):
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.mesh.order import renumber
    m = bump_channel(7, 4, 3, amplitude=0.05, seed=1)
    r = renumber(m.nodes, m.elements, ordering)
    assert sorted(r.node_perm) == list(range(m.n_nodes))
    assert sorted(r.elem_perm) == list(range(m.n_tets))
    # each element keeps its nodes and their local order
    assert np.array_equal(r.nodes[r.elements], m.nodes[m.elements[r.elem_perm]])
    a = np.arange(m.n_nodes) * 1.5
    assert np.array_equal(r.nodal_back(r.nodal(a)), a)
    assert np.array_equal(r.elemental_back(r.elemental(np.arange(m.n_tets))), np.arange(m.n_tets))
    assert np.array_equal(r.element_ids_back(r.elem_inv), np.arange(m.n_tets))
    d_new = r.node_set(m.dirichlet_nodes)
    assert np.array_equal(np.sort(r.node_perm[d_new]), np.sort(m.dirichlet_nodes))
    if ordering == "given":
        assert np.array_equal(r.elements, m.elements)


def test_unknown_ordering_raises():
    from up3d_b200.mesh.order import renumber
    with pytest.raises(ValueError):
        renumber(np.zeros((4, 3)), np.array([[0, 1, 2, 3]]), "rcm")


def test_choking_mach_of_the_bump_channel():
    """Quasi-1-D choking estimate: the configurations' bumps choke the
    channel at M 0.7685 (bump 0.05) and M 0.7105 (bump 0.08); a vanishing
    bump chokes only at M 1."""
    from up3d_b200.mesh.kuhn import choking_mach
    assert abs(choking_mach(0.05) - 0.76850) < 1e-4
    assert abs(choking_mach(0.08) - 0.71049) < 1e-4
    assert choking_mach(0.0) == 1.0
    assert choking_mach(1e-4) > 0.98
