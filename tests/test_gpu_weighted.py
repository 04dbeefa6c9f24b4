"""The weighted upwind modes on the device (kernels/upwind.py:128-454):
face normals, the BFS neighbourhoods and the "kernel" / "blend" upwinded
densities against the reference's outputs (tests/golden/weighted_upwind.npz)
and the oracle, plus the invariants of the reference's own tests
(tests/test_p6_weighted_flux.py, tests/test_p7_diff_flux.py)."""

import numpy as np
import pytest

from conftest import GOLDEN, REL_TOL, has_cuda, rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]

M_CRIT, UPWIND_C, RHO_FLOOR, M_CAP, GAMMA = 0.95, 1.5, 0.05, 3.0, 1.4
PARAMS = {
    "default": dict(p_weight=3.0, reach_frac=1.0, reach_gain_max=4.0, nbr_depth=3,
                    sigma_s_frac=0.35, sigma_p_frac=0.35),
    "alt": dict(p_weight=2.0, reach_frac=0.8, reach_gain_max=3.0, nbr_depth=2,
                sigma_s_frac=0.5, sigma_p_frac=0.25),
}


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "weighted_upwind.npz")


def _states(gold):
    return sorted({k.split("/")[1] for k in gold.files if k.startswith("state/")})


def _inputs(nodes, elements, phi, m_inf):
    from oracle import oracle as O
    op = O.PicardOperator(nodes, elements)
    grad, q2 = op.velocities(phi)
    q2l = O.limit_q2_field(q2, m_inf, M_CAP, GAMMA)
    return grad.copy(), q2l, O.density_field(q2l, m_inf, GAMMA)


def test_face_normals_match_reference(gold):
    from up3d_b200.kernels.upwind import compute_face_normals
    nodes, elements = gold["mesh/nodes"], gold["mesh/elements"]
    out = np.empty((len(elements), 4, 3))
    compute_face_normals(nodes, elements, out)
    assert np.abs(out - gold["mesh/face_normals"]).max() < 1e-14


@pytest.mark.parametrize("pname", ["default", "alt"])
def test_neighborhoods_match_reference_exactly(gold, pname):
    from up3d_b200.kernels.upwind import UpwindOperator, build_upstream_neighborhoods
    nodes, elements = gold["mesh/nodes"], gold["mesh/elements"]
    upw = UpwindOperator(nodes, elements, weighted=True, mode="kernel", **PARAMS[pname])
    assert np.array_equal(upw._nb_off, gold[f"{pname}/nb_off"])
    assert np.array_equal(upw._nb_idx, gold[f"{pname}/nb_idx"])
    off, idx = build_upstream_neighborhoods(upw.face_neighbors, PARAMS[pname]["nbr_depth"])
    assert np.array_equal(off, gold[f"{pname}/nb_off"]) and np.array_equal(idx, gold[f"{pname}/nb_idx"])


@pytest.mark.parametrize("pname", ["default", "alt"])
@pytest.mark.parametrize("mode", ["kernel", "blend"])
def test_weighted_rho_tilde_matches_reference(gold, pname, mode):
    from up3d_b200.kernels.upwind import UpwindOperator
    nodes, elements = gold["mesh/nodes"], gold["mesh/elements"]
    upw = UpwindOperator(nodes, elements, weighted=True, mode=mode, **PARAMS[pname])
    for label in _states(gold):
        phi, m_inf = gold[f"state/{label}/phi"], float(gold[f"state/{label}/m_inf"])
        grad, q2l, rho = _inputs(nodes, elements, phi, m_inf)
        rt = upw.rho_tilde(grad, q2l, rho, m_inf, UPWIND_C, M_CRIT, GAMMA, RHO_FLOOR).copy()
        key = f"{pname}/{mode}/{label}"
        assert rel_err(rt, gold[f"{key}/rho_tilde"]) < REL_TOL, key
        assert rel_err(upw.nu, gold[f"{key}/nu"]) < REL_TOL, key
        assert upw.n_supersonic == int(gold[f"{key}/n_supersonic"]), key
        assert upw.n_floored == int(gold[f"{key}/n_floored"]), key
        assert abs(upw.nu_max - float(gold[f"{key}/nu_max"])) <= 1e-12 * max(1.0, upw.nu_max), key


@pytest.mark.parametrize("depth", [1, 2, 3, 4, 5, 7])
def test_neighborhoods_match_oracle_on_a_larger_mesh(depth):
    from oracle import oracle as O
    from up3d_b200.kernels.upwind import build_upstream_neighborhoods
    from up3d_b200.mesh.kuhn import bump_channel
    m = bump_channel(12, 5, 4, amplitude=0.05, seed=2)
    fn = O.face_adjacency(m.elements)
    ref_off, ref_idx = O.build_upstream_neighborhoods(fn, depth)
    off, idx = build_upstream_neighborhoods(fn, depth)
    assert np.array_equal(off, ref_off) and np.array_equal(idx, ref_idx)


@pytest.mark.parametrize("mode", ["kernel", "blend"])
def test_weighted_rho_tilde_matches_oracle_on_pocket_states(mode):
    import torch
    from oracle import oracle as O
    from up3d_b200.kernels.upwind import UpwindOperator
    from up3d_b200.mesh.kuhn import bump_channel, pocket_state
    m = bump_channel(30, 10, 9, amplitude=0.08, seed=2)
    ref = O.UpwindOperator(m.nodes, m.elements, weighted=True, mode=mode)
    upw = UpwindOperator(m.nodes, m.elements, weighted=True, mode=mode)
    for fam in ("accelerating", "shockpoint", "mixed"):
        grad, q2l, rho = _inputs(m.nodes, m.elements, pocket_state(m, fam), 0.8)
        r = ref.rho_tilde(grad, q2l, rho, 0.8, UPWIND_C, M_CRIT).copy()
        # device tensors in, device views out
        d = upw.rho_tilde(torch.from_numpy(grad).cuda(), torch.from_numpy(q2l).cuda(),
                          torch.from_numpy(rho).cuda(), 0.8, UPWIND_C, M_CRIT)
        assert d.is_cuda
        assert rel_err(d.cpu().numpy(), r) < REL_TOL, fam
        nu = upw.nu  # host copy: the operator was built on host arrays
        assert rel_err(nu.cpu().numpy() if hasattr(nu, "cpu") else nu, ref.nu) < REL_TOL, fam
        assert upw.n_supersonic == ref.n_supersonic and upw.n_floored == ref.n_floored
        assert ref.n_supersonic > 0


def _cube_like():
    from up3d_b200.mesh.kuhn import bump_channel
    m = bump_channel(6, 6, 6, amplitude=0.0, seed=0)
    return m.nodes, m.elements


def test_subcritical_noop_bitwise_and_uniform_density_invariant():
    from oracle import oracle as O
    from up3d_b200.kernels.upwind import UpwindOperator
    nodes, elements = _cube_like()
    upw = UpwindOperator(nodes, elements, weighted=True, mode="kernel")
    grad, q2, rho = _inputs(nodes, elements, nodes[:, 0].copy(), 0.5)
    rt = upw.rho_tilde(grad, q2, rho, 0.5, UPWIND_C, M_CRIT)
    assert upw.nu_max == 0.0
    assert np.array_equal(rt, rho)                     # bit-exact no-op
    phi = 1.3 * nodes[:, 0]
    grad, q2 = O.PicardOperator(nodes, elements).velocities(phi)
    assert O.mach_squared_field(q2, 0.8).max() > M_CRIT ** 2
    rho = np.full(len(elements), 0.7)
    for mode in ("kernel", "blend"):
        u = UpwindOperator(nodes, elements, weighted=True, mode=mode)
        rt = u.rho_tilde(grad, q2, rho, 0.8, UPWIND_C, M_CRIT)
        assert u.nu_max > 0.0
        assert np.allclose(rt, 0.7, atol=1e-12)        # a convex blend of a uniform field


def test_weighted_sweep_deterministic_and_floored():
    from up3d_b200.kernels.upwind import UpwindOperator
    nodes, elements = _cube_like()
    phi = 1.2 * nodes[:, 0] + 0.15 * nodes[:, 0] ** 2
    grad, q2, rho = _inputs(nodes, elements, phi, 0.85)
    for mode in ("kernel", "blend"):
        upw = UpwindOperator(nodes, elements, weighted=True, mode=mode)
        a = upw.rho_tilde(grad, q2, rho, 0.85, UPWIND_C, M_CRIT).copy()
        b = upw.rho_tilde(grad, q2, rho, 0.85, UPWIND_C, M_CRIT).copy()
        assert np.all(np.isfinite(a)) and np.array_equal(a, b)
        assert a.min() >= RHO_FLOOR - 1e-15


def test_weighted_mode_offers_rho_tilde_only_and_walk_mode_is_unchanged():
    from oracle import oracle as O
    from up3d_b200.kernels.upwind import UpwindOperator
    nodes, elements = _cube_like()
    grad, q2, rho = _inputs(nodes, elements, 1.25 * nodes[:, 0], 0.82)
    w = UpwindOperator(nodes, elements, weighted=True, mode="kernel")
    with pytest.raises(NotImplementedError):
        w.rho_tilde_sensitivities(grad, q2, rho, 0.82, UPWIND_C, M_CRIT)
    with pytest.raises(NotImplementedError):
        w.freeze_upwind_state(grad, q2, rho, 0.82, UPWIND_C, M_CRIT)
    walk = UpwindOperator(nodes, elements, weighted=False).rho_tilde(grad, q2, rho, 0.82, UPWIND_C, M_CRIT)
    ref = O.UpwindOperator(nodes, elements).rho_tilde(grad, q2, rho, 0.82, UPWIND_C, M_CRIT)
    assert rel_err(walk, ref) < REL_TOL
    with pytest.raises(ValueError, match="depth"):
        UpwindOperator(nodes, elements, weighted=True, mode="kernel", nbr_depth=0)


def test_kernel_mode_deeper_than_four_hops_matches_oracle():
    """Neighbourhoods past four hops (built on the host) feed the same
    kernel-mode sweep: the oracle's rho~ at nbr_depth 5 and 6."""
    from oracle import oracle as O
    from up3d_b200.kernels.upwind import UpwindOperator
    from up3d_b200.mesh.kuhn import bump_channel, pocket_state
    m = bump_channel(16, 6, 5, amplitude=0.08, seed=2)
    grad, q2l, rho = _inputs(m.nodes, m.elements, pocket_state(m, "mixed"), 0.8)
    for depth in (5, 6):
        ref = O.UpwindOperator(m.nodes, m.elements, weighted=True, mode="kernel", nbr_depth=depth)
        upw = UpwindOperator(m.nodes, m.elements, weighted=True, mode="kernel", nbr_depth=depth)
        r = ref.rho_tilde(grad, q2l, rho, 0.8, UPWIND_C, M_CRIT).copy()
        d = upw.rho_tilde(grad, q2l, rho, 0.8, UPWIND_C, M_CRIT)
        assert rel_err(d, r) < REL_TOL, depth
        assert upw.n_supersonic == ref.n_supersonic, depth


def test_masked_face_neighbors_rebuild_the_neighborhoods():
    from oracle import oracle as O
    from up3d_b200.kernels.upwind import UpwindOperator
    from up3d_b200.mesh.kuhn import bump_channel, pocket_state
    m = bump_channel(12, 5, 4, amplitude=0.05, seed=3)
    upw = UpwindOperator(m.nodes, m.elements, weighted=True, mode="kernel")
    fn = np.array(upw.face_neighbors)
    fn[::7, 1] = -1                                    # cut some faces (a wake-style mask)
    upw.face_neighbors = fn
    ref_off, ref_idx = O.build_upstream_neighborhoods(fn, 3)
    assert np.array_equal(upw._nb_off, ref_off) and np.array_equal(upw._nb_idx, ref_idx)
    ref = O.UpwindOperator(m.nodes, m.elements, weighted=True, mode="kernel")
    ref.face_neighbors = fn
    ref._nb_off, ref._nb_idx = ref_off, ref_idx
    grad, q2, rho = _inputs(m.nodes, m.elements, pocket_state(m, "mixed"), 0.8)
    assert rel_err(upw.rho_tilde(grad, q2, rho, 0.8, UPWIND_C, M_CRIT),
                   ref.rho_tilde(grad, q2, rho, 0.8, UPWIND_C, M_CRIT)) < REL_TOL
