"""The level-set path's per-side pieces in the oracle against the
reference (tests/golden/side_terms.npz): the walk and rho~ on a face graph
restricted to one side, and newton_terms23_side_coo."""

import numpy as np
import pytest

from conftest import GOLDEN, REL_TOL, rel_err


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "side_terms.npz")


def _state(gold):
    from oracle import oracle as O
    nodes, el = gold["nodes"], gold["elements"]
    op = O.PicardOperator(nodes, el)
    grad, q2 = op.velocities(gold["phi"])
    q2l = O.limit_q2_field(q2, 0.8, 3.0)
    return op, grad.copy(), q2l, O.density_field(q2l, 0.8)


@pytest.mark.parametrize("label", ["upper", "lower"])
def test_side_restricted_walk(gold, label):
    from oracle import oracle as O
    nodes, el = gold["nodes"], gold["elements"]
    _, grad, q2l, rho = _state(gold)
    keep = gold[f"{label}/keep"]
    upw = O.UpwindOperator(nodes, el)
    fn = upw.face_neighbors.copy()
    nb_ok = np.where(fn >= 0, keep[np.clip(fn, 0, None)], False)
    fn[~(nb_ok & keep[:, None])] = -1
    assert np.array_equal(fn, gold[f"{label}/fn"])
    upw.face_neighbors = fn
    rt = upw.rho_tilde(grad, q2l, rho, 0.8, 1.5, 0.95)
    assert np.array_equal(upw._upstream, gold[f"{label}/upstream"])
    assert rel_err(rt, gold[f"{label}/rho_tilde"]) < REL_TOL


def test_newton_terms23_side_coo(gold):
    from oracle import oracle as O
    op, _, _, _ = _state(gold)
    side = {k[4:]: gold[k] for k in gold.files if k.startswith("t23/") and k not in
            ("t23/rows", "t23/cols", "t23/data")}
    rows, cols, data = O.newton_terms23_side_coo(op.B, op.V, side, u_inf=1.3)
    assert np.array_equal(rows, gold["t23/rows"]) and np.array_equal(cols, gold["t23/cols"])
    assert np.abs(data - gold["t23/data"]).max() <= 1e-14 * np.abs(gold["t23/data"]).max()
