"""The oracle's wall force post-processing (tangential gradients, outward
normals, edge adjacency, smoothing, Cp, force coefficients) against the
reference's post/surface.py on the channel's lower wall
(tests/golden/wall_forces.npz)."""

import numpy as np
import pytest

from conftest import GOLDEN


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "wall_forces.npz")


def test_wall_geometry(gold):
    from oracle import oracle as O
    nodes, el, wf = gold["nodes"], gold["elements"], gold["wall_faces"]
    _, area, tn = O.wall_tri_gradients(nodes, wf, nodes[:, 0])
    assert np.abs(area - gold["area"]).max() <= 1e-15 * area.max()
    assert np.abs(tn - gold["tri_normal"]).max() <= 1e-15
    assert np.abs(O.wall_outward_normals(nodes, el, wf) - gold["out_normal"]).max() <= 1e-15
    assert np.array_equal(O.wall_adjacency(wf), gold["adjacency"])


def test_wall_forces(gold):
    from oracle import oracle as O
    nodes, el, wf = gold["nodes"], gold["elements"], gold["wall_faces"]
    labels = sorted({k.split("/")[0] for k in gold.files if "/" in k})
    for label in labels:
        phi, m = gold[f"{label}/phi"], float(gold[f"{label}/m_inf"])
        g, _, _ = O.wall_tri_gradients(nodes, wf, phi)
        assert np.abs(g - gold[f"{label}/grad"]).max() <= 1e-13 * np.abs(gold[f"{label}/grad"]).max()
        for alpha in (0, 4):
            for sp_ in (0, 2):
                q = f"{label}/a{alpha}_s{sp_}/"
                r = O.wall_force_coefficients(nodes, el, wf, phi, alpha_deg=alpha, s_ref=2.5, m_inf=m,
                                              smooth_passes=sp_)
                cp = gold[q + "cp_tri"]
                assert np.abs(r["cp_tri"] - cp).max() <= 1e-12 * max(1.0, np.abs(cp).max()), q
                scale = np.abs(cp).max() * 1.0
                assert np.abs(r["cf"] - gold[q + "cf"]).max() <= 1e-12 * scale, q
                assert abs(r["cl"] - float(gold[q + "cl"])) <= 1e-12 * scale, q
                assert abs(r["cd_pressure"] - float(gold[q + "cd"])) <= 1e-12 * scale, q
