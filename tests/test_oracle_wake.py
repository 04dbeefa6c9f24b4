"""The oracle's wake master-slave elimination and Kutta targets against
the reference's own WakeConstraint / kutta_targets on synthetic plane-sheet
cuts of the channel (tests/golden/wake_constraint.npz), and the synthetic
cut's structure."""

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "wake_constraint.npz")


def _cut(single):
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.mesh.wake_cut import cut_channel_sheet
    return cut_channel_sheet(bump_channel(10, 4, 4, amplitude=0.08, seed=1), single_station=single)


def _csr(g, q, n_rows, n_cols):
    return sp.csr_matrix((g[q + "data"], g[q + "indices"], g[q + "indptr"]), shape=(n_rows, n_cols))


@pytest.mark.parametrize("tag", ["multi", "single"])
@pytest.mark.parametrize("mat", ["picard", "newton"])
def test_oracle_wake_constraint_matches_reference(gold, tag, mat):
    from oracle import oracle as O
    cut = _cut(tag == "single")
    assert np.array_equal(cut.nodes, gold[f"{tag}/nodes"])
    assert np.array_equal(cut.elements, gold[f"{tag}/elements"])
    q = f"{tag}/{mat}/"
    n_cut = len(cut.nodes)
    A = _csr(gold, q + "A_", n_cut, n_cut)
    con = O.WakeConstraint(A, cut.wc)
    n_red, n_st = con.n_reduced, cut.wc.n_stations
    ref_red = _csr(gold, q + "red_", n_red, n_red)
    ref_H = _csr(gold, q + "H_", n_red, n_st)
    A_red, H = con.reduce_operator(A)
    scale = np.abs(ref_red.data).max()
    assert np.array_equal(A_red.indptr, ref_red.indptr) and np.array_equal(A_red.indices, ref_red.indices)
    assert np.abs(A_red.data - ref_red.data).max() <= 1e-14 * scale
    assert np.array_equal(H.indptr, ref_H.indptr) and np.array_equal(H.indices, ref_H.indices)
    assert np.abs(H.data - ref_H.data).max() <= 1e-14 * scale
    assert np.abs(con._h - gold[q + "h_dense"]).max() <= 1e-14 * scale
    rhs = con.reduced_rhs(gold[q + "b"], gold[q + "gamma"])
    assert np.abs(rhs - gold[q + "rhs"]).max() <= 1e-13 * np.abs(gold[q + "rhs"]).max()
    assert np.array_equal(con.expand(gold[q + "phi_red"], gold[q + "gamma"]), gold[q + "expand"])


@pytest.mark.parametrize("tag", ["multi", "single"])
def test_oracle_kutta_targets_match_reference(gold, tag):
    from oracle import oracle as O
    cut = _cut(tag == "single")
    k = O.kutta_targets(gold[f"{tag}/phi_cut"], cut.wc)
    assert np.abs(k - gold[f"{tag}/kutta"]).max() <= 1e-15


def test_synthetic_cut_structure():
    cut = _cut(False)
    wc = cut.wc
    n = wc.n_nodes_orig
    assert np.array_equal(wc.slave_nodes, n + np.arange(len(wc.slave_nodes)))
    assert np.array_equal(cut.nodes[wc.slave_nodes], cut.nodes[wc.master_nodes])
    # every node is referenced; the slaves only by "+"-side elements
    assert len(np.unique(cut.elements)) == len(cut.nodes)
    uses_slave = np.any(cut.elements >= n, axis=1)
    uses_master = np.isin(cut.elements, wc.master_nodes).any(axis=1)
    assert uses_slave.sum() > 0 and (uses_master & ~uses_slave).sum() > 0
    assert wc.n_stations == 5 and set(wc.node_station) == set(range(5))
