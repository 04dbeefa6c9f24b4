"""Wall Cp and pressure forces on the device (post/surface.py:80-363)
against the reference (tests/golden/wall_forces.npz) and the oracle."""

import numpy as np
import pytest

from conftest import GOLDEN, has_cuda

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "wall_forces.npz")


def test_wall_geometry_matches_reference(gold):
    from up3d_b200.post.surface import triangle_tangential_gradients, wall_outward_normals
    nodes, el, wf = gold["nodes"], gold["elements"], gold["wall_faces"]
    _, area, tn = triangle_tangential_gradients(nodes, wf, nodes[:, 0].copy(), elements=el)
    assert np.abs(area - gold["area"]).max() <= 1e-15 * area.max()
    assert np.abs(tn - gold["tri_normal"]).max() <= 1e-15
    assert np.abs(wall_outward_normals(nodes, el, wf) - gold["out_normal"]).max() <= 1e-15


def test_wall_forces_match_reference(gold):
    from up3d_b200.post.surface import triangle_tangential_gradients, wall_force_coefficients
    nodes, el, wf = gold["nodes"], gold["elements"], gold["wall_faces"]
    labels = sorted({k.split("/")[0] for k in gold.files if "/" in k})
    for label in labels:
        phi, m = gold[f"{label}/phi"], float(gold[f"{label}/m_inf"])
        g, _, _ = triangle_tangential_gradients(nodes, wf, phi, elements=el)
        assert np.abs(g - gold[f"{label}/grad"]).max() <= 1e-13 * np.abs(gold[f"{label}/grad"]).max()
        for alpha in (0, 4):
            for sp_ in (0, 2):
                q = f"{label}/a{alpha}_s{sp_}/"
                r = wall_force_coefficients(nodes, el, wf, phi, alpha_deg=alpha, s_ref=2.5, m_inf=m,
                                            smooth_passes=sp_)
                cp = gold[q + "cp_tri"]
                scale = max(1.0, np.abs(cp).max())
                assert np.abs(r["cp_tri"] - cp).max() <= 1e-12 * scale, q
                assert np.abs(r["cf"] - gold[q + "cf"]).max() <= 1e-12 * scale, q
                assert abs(r["cl"] - float(gold[q + "cl"])) <= 1e-12 * scale, q
                assert abs(r["cd_pressure"] - float(gold[q + "cd"])) <= 1e-12 * scale, q


def test_wall_forces_device_inputs_and_larger_mesh_match_oracle():
    import torch
    from oracle import oracle as O
    from up3d_b200.adjoint import lower_wall_faces
    from up3d_b200.mesh.kuhn import bump_channel, pocket_state
    from up3d_b200.post.surface import wall_force_coefficients
    m = bump_channel(60, 20, 10, amplitude=0.08, seed=5)
    wf = lower_wall_faces(m.elements, m.shape)[:, 1:]
    phi = pocket_state(m, "mixed")
    for sp_ in (0, 3):
        ref = O.wall_force_coefficients(m.nodes, m.elements, wf, phi, alpha_deg=2.0, s_ref=1.7, m_inf=0.8,
                                        smooth_passes=sp_)
        r = wall_force_coefficients(m.nodes, m.elements, wf, torch.from_numpy(phi).cuda(), alpha_deg=2.0,
                                    s_ref=1.7, m_inf=0.8, smooth_passes=sp_)
        assert r["cp_tri"].is_cuda
        scale = np.abs(ref["cp_tri"]).max()
        assert np.abs(r["cp_tri"].cpu().numpy() - ref["cp_tri"]).max() <= 1e-12 * scale
        assert np.abs(r["cf"] - ref["cf"]).max() <= 1e-12 * scale * len(wf) ** 0.5
        # deterministic: the force sum has a fixed order
        r2 = wall_force_coefficients(m.nodes, m.elements, wf, torch.from_numpy(phi).cuda(), alpha_deg=2.0,
                                     s_ref=1.7, m_inf=0.8, smooth_passes=sp_)
        assert np.array_equal(r2["cf"], r["cf"])


def test_unowned_wall_face_raises():
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.post.surface import wall_force_coefficients
    m = bump_channel(6, 3, 3, amplitude=0.0, seed=0)
    bad = np.array([[0, 1, 2]], dtype=np.int64)   # not a face of any tet
    with pytest.raises(ValueError, match="owned"):
        wall_force_coefficients(m.nodes, m.elements, bad, m.freestream())


def test_mesh_handle_lookup_by_identity_sees_in_place_changes():
    """get_mesh finds the handle of tensors (and read-only arrays) it has
    seen by identity; an in-place change of a tensor (its version counter)
    or a writeable array (its digest) gives the changed mesh's handle."""
    import torch
    from up3d_b200.mesh.device import get_mesh
    from up3d_b200.mesh.kuhn import bump_channel
    m = bump_channel(6, 3, 3, amplitude=0.05, seed=0)
    nodes_d = torch.from_numpy(m.nodes.copy()).cuda()
    elements_d = torch.from_numpy(m.elements.copy()).cuda()
    a = get_mesh(nodes_d, elements_d)
    assert get_mesh(nodes_d, elements_d) is a
    assert get_mesh(m.nodes, m.elements) is a            # same contents, by digest
    nodes_d[0, 0] += 0.25
    b = get_mesh(nodes_d, elements_d)
    assert b is not a and np.allclose(b.nodes[0, 0], m.nodes[0, 0] + 0.25)
    ro_n, ro_e = m.nodes.copy(), m.elements.copy()
    ro_n.flags.writeable = False
    ro_e.flags.writeable = False
    assert get_mesh(ro_n, ro_e) is a and get_mesh(ro_n, ro_e) is a
    w = m.nodes.copy()
    assert get_mesh(w, m.elements) is a
    w[1, 1] += 0.5
    assert get_mesh(w, m.elements) is not a
