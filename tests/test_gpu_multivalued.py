"""The level-set MultivaluedOperator over the device operators against the
reference (tests/golden/multivalued.npz from pyfp3d/wake/multivalued.py):
the extended matrices of both closures, the per-side upwinded densities
(per-side walks on own-side face graphs) with their monitors, and the
per-side Newton records live and frozen, at M0.8 with a jump on the aux
DOFs; floating point within 1e-12 of the largest magnitude, selections and
masks exactly."""

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN, has_cuda, rel_err, sparse_rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]

M_INF, C, M_CRIT = 0.8, 1.5, 0.95


@pytest.fixture(scope="module")
def mv():
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.wake import CutElementMap, MultivaluedOperator, WakeLevelSet
    g = np.load(GOLDEN / "multivalued.npz")
    mesh = bump_channel(16, 6, 5, amplitude=0.08, seed=3)
    ls = WakeLevelSet(g["te_points"], g["direction"])
    cm = CutElementMap(mesh.nodes, mesh.elements, ls)
    return g, MultivaluedOperator(mesh.nodes, mesh.elements, cm, levelset=ls)


def _csr(g, tag, n):
    return sp.csr_matrix((g[tag + "/data"], g[tag + "/indices"], g[tag + "/indptr"]), shape=(n, n))


def test_extended_matrices(mv):
    g, op = mv
    n = op.n_total
    assert sparse_rel_err(op.assemble_matrix(None).to_scipy(), _csr(g, "A_laplace", n)) < 1e-12
    assert sparse_rel_err(op.assemble_matrix(g["rho_main"]).to_scipy(), _csr(g, "A_continuity", n)) < 1e-12
    ru, rl = op.element_densities(g["phi_ext"], M_INF)
    assert rel_err(ru, g["rho_up"]) < 1e-12 and rel_err(rl, g["rho_lo"]) < 1e-12
    A = op.assemble_matrix((ru, rl), closure="wake_ls", te_kutta="mass")
    assert sparse_rel_err(A.to_scipy(), _csr(g, "A_wake_ls", n)) < 1e-12
    # no TE nodes on this sheet: the pressure Kutta form is the mass form
    A2 = op.assemble_matrix((ru, rl), closure="wake_ls")
    assert sparse_rel_err(A2.to_scipy(), _csr(g, "A_wake_ls", n)) < 1e-12


def test_per_side_densities_and_monitors(mv):
    g, op = mv
    up, lo = op.side_potentials(g["phi_ext"])
    assert np.array_equal(up, g["phi_up"]) and np.array_equal(lo, g["phi_lo"])
    nodes = np.flatnonzero(op.cm.ext_dof_of_node >= 0)
    assert np.array_equal(op.node_jump(g["phi_ext"], nodes), g["node_jump"])
    rt_u, rt_l = op.element_rho_tilde(g["phi_ext"], M_INF, C, M_CRIT)
    assert rel_err(rt_u, g["rt_up"]) < 1e-12 and rel_err(rt_l, g["rt_lo"]) < 1e-12
    mon = g["mon"]
    assert op.n_nu_active == int(mon[1]) and op.n_floored == int(mon[2]) and op.n_limited == int(mon[3])
    assert abs(op.nu_max - mon[0]) <= 1e-12 * max(abs(mon[0]), 1.0)
    assert op.n_nu_active > 100
    assert np.array_equal(op.nu_active_elements(), g["nu_active_elements"])
    assert rel_err(op.element_mach2(g["phi_ext"], M_INF), g["mach2"]) < 1e-12


@pytest.mark.parametrize("tag", ["live", "frozen"])
def test_per_side_newton_records(mv, tag):
    g, op = mv
    frozen = None
    if tag == "frozen":
        frozen = op.freeze_side_state(g["phi_ext"], M_INF, C, M_CRIT)
        for k, side in enumerate(("upper", "lower")):
            assert np.array_equal(frozen[k][0], g[f"freeze/{side}/upstream"])
            assert np.array_equal(frozen[k][1], g[f"freeze/{side}/branch"])
    recs = op.newton_side_data(g["phi_ext"], M_INF, C, M_CRIT, frozen=frozen)
    for side, rec in zip(("upper", "lower"), recs):
        p = f"{tag}/{side}/"
        for key in ("upstream", "lim_mask", "keep", "dofvec", "readvec"):
            assert np.array_equal(np.asarray(rec[key]), g[p + key]), (side, key)
        for key in ("rho_tilde", "s_e", "s_u", "grad", "grad_row"):
            assert rel_err(np.asarray(rec[key]), g[p + key]) < 1e-12, (side, key)
    mon = g[f"{tag}/mon"]
    assert op.n_nu_active == int(mon[1]) and op.n_floored == int(mon[2]) and op.n_limited == int(mon[3])


def test_device_inputs_stay_on_the_device(mv):
    import torch
    g, op = mv
    phi = torch.from_numpy(g["phi_ext"]).cuda()
    rt_u, rt_l = op.element_rho_tilde(phi, M_INF, C, M_CRIT)
    assert rt_u.is_cuda and rel_err(rt_u.cpu().numpy(), g["rt_up"]) < 1e-12
    rec_u, _ = op.newton_side_data(phi, M_INF, C, M_CRIT)
    assert rec_u["s_e"].is_cuda


def test_unbuilt_options_raise(mv):
    from up3d_b200.wake import MultivaluedOperator
    g, op = mv
    with pytest.raises(NotImplementedError):
        op.assemble_matrix(None, closure="nope")
    with pytest.raises(NotImplementedError):
        op.assemble_matrix(None, closure="wake_ls", tip_taper=np.full(3, 0.5))
    with pytest.raises(NotImplementedError):
        MultivaluedOperator(op.nodes, op.elements, op.cm, span_blend=("cos", 0.1))
    with pytest.raises(ValueError):
        MultivaluedOperator(op.nodes, op.elements, op.cm).assemble_matrix(None, closure="wake_ls")
