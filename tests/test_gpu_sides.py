"""The level-set path's per-side pieces on the device against the reference
(tests/golden/side_terms.npz) and the oracle: the walk and rho~ on a face
graph restricted to one side's elements, and newton_terms23_side_coo."""

import numpy as np
import pytest

from conftest import GOLDEN, REL_TOL, has_cuda, rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "side_terms.npz")


def _state(nodes, el, phi, m=0.8):
    from oracle import oracle as O
    grad, q2 = O.PicardOperator(nodes, el).velocities(phi)
    q2l = O.limit_q2_field(q2, m, 3.0)
    return grad.copy(), q2l, O.density_field(q2l, m)


@pytest.mark.parametrize("label", ["upper", "lower"])
def test_side_restricted_walk_matches_reference(gold, label):
    from up3d_b200.kernels.upwind import UpwindOperator
    nodes, el = gold["nodes"], gold["elements"]
    grad, q2l, rho = _state(nodes, el, gold["phi"])
    keep = gold[f"{label}/keep"]
    upw = UpwindOperator(nodes, el)
    fn = np.array(upw.face_neighbors)
    nb_ok = np.where(fn >= 0, keep[np.clip(fn, 0, None)], False)
    fn[~(nb_ok & keep[:, None])] = -1
    upw.face_neighbors = np.ascontiguousarray(fn)
    rt = upw.rho_tilde(grad, q2l, rho, 0.8, 1.5, 0.95)
    assert np.array_equal(upw.upstream(grad), gold[f"{label}/upstream"])
    assert rel_err(rt, gold[f"{label}/rho_tilde"]) < REL_TOL
    assert rel_err(upw.nu, gold[f"{label}/nu"]) < REL_TOL
    # the unmasked operator on the same mesh is unaffected (the masked one forked the handle)
    plain = UpwindOperator(nodes, el)
    assert (np.asarray(plain.face_neighbors) >= 0).sum() > (fn >= 0).sum()


def _side(gold):
    return {k[4:]: gold[k] for k in gold.files
            if k.startswith("t23/") and k not in ("t23/rows", "t23/cols", "t23/data")}


def test_newton_terms23_side_coo_matches_reference(gold):
    import torch
    from up3d_b200.kernels.cut_assembly import newton_terms23_side_coo
    from up3d_b200.kernels.jacobian import PicardOperator
    op = PicardOperator(gold["nodes"], gold["elements"])
    side = _side(gold)
    rows, cols, data = newton_terms23_side_coo(op, side, u_inf=1.3)
    assert np.array_equal(rows, gold["t23/rows"]) and np.array_equal(cols, gold["t23/cols"])
    assert np.abs(data - gold["t23/data"]).max() <= 1e-14 * np.abs(gold["t23/data"]).max()
    # device inputs give device outputs, the same triplets; no readvec / grad_row -> dofvec / grad
    dside = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in side.items()}
    r2, c2, d2 = newton_terms23_side_coo(op, dside, u_inf=1.3)
    assert r2.is_cuda and np.array_equal(d2.cpu().numpy(), data)
    from oracle import oracle as O
    bare = {k: v for k, v in side.items() if k not in ("readvec", "grad_row")}
    ref = O.newton_terms23_side_coo(O.PicardOperator(gold["nodes"], gold["elements"]).B,
                                    O.PicardOperator(gold["nodes"], gold["elements"]).V, bare, u_inf=1.3)
    r3, c3, d3 = newton_terms23_side_coo(op, bare, u_inf=1.3)
    assert np.array_equal(r3, ref[0]) and np.array_equal(c3, ref[1])
    assert np.abs(d3 - ref[2]).max() <= 1e-14 * np.abs(ref[2]).max()


def test_side_coo_rejects_bad_upstream(gold):
    from up3d_b200.kernels.cut_assembly import newton_terms23_side_coo
    from up3d_b200.kernels.jacobian import PicardOperator
    op = PicardOperator(gold["nodes"], gold["elements"])
    side = _side(gold)
    side["upstream"] = side["upstream"].copy()
    side["upstream"][3] = len(gold["elements"]) + 5
    with pytest.raises(ValueError, match="upstream"):
        newton_terms23_side_coo(op, side)
