"""Launch shapes of the fused evaluation.  The two-pass form (element sweep
+ row gather): every shape (one thread per element or a persistent wave;
4-32 lanes per row) gives the same bits.  The tiled form: each tile size
gives its own fixed summation order (bit-reproducible, residual-only and
Jacobian evaluations agree bitwise) and agrees with the two-pass form and
the oracle to rounding.  The autotuner installs one of the listed forms and
bad shapes are refused."""

import numpy as np
import pytest

from conftest import has_cuda, rel_err, sparse_rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]

# (persistent, resident threads per SM, lanes per row, fixed-width gather
# records) of the two-pass form
SHAPES = [(0, 512, 4, 0), (0, 768, 8, 1), (1, 512, 8, 0), (1, 768, 16, 1), (1, 640, 32, 0), (0, 640, 4, 1),
          (1, 640, 16, 1), (1, 640, 8, 1)]


def _setup():
    import torch
    from up3d_b200.mesh.device import DeviceMesh
    from up3d_b200.mesh.kuhn import bump_channel, pocket_state
    from up3d_b200.solve.fused import ResidualJacobian
    # 30x10x9 hexes: 16,200 tets, not a multiple of the 256-element tile
    mesh = bump_channel(30, 10, 9, amplitude=0.08, seed=2)
    phi_h = pocket_state(mesh, "mixed")
    dm = DeviceMesh(mesh.nodes, mesh.elements)
    return mesh, phi_h, dm, ResidualJacobian(dm), torch.from_numpy(phi_h).cuda()


def _outputs(ev, phi, flow, frozen=None):
    R = ev.evaluate(phi, flow, jacobian=True, frozen=frozen).clone()
    J = ev.jacobian().to_scipy()
    return R, J, ev.upstream.clone(), ev.rho_tilde.clone(), ev.read_monitors()


def test_every_shape_gives_the_same_bits():
    import torch
    from up3d_b200.solve.fused import FlowParams
    mesh, phi_h, dm, ev, phi = _setup()
    assert dm.n_tets % 256 != 0
    flow = FlowParams(m_inf=0.8)
    t0 = dm.tuning()
    assert t0["row_lanes"] == 8 and t0["elem_persistent"] == 0 and t0["elem_threads_per_sm"] == 512
    assert t0["assembly"] == 0 and t0["tile_elems"] == 256 and t0["tile_stretch"] == 1
    dm.set_tuning(*SHAPES[0], assembly=0)
    R0, J0, up0, rt0, mon0 = _outputs(ev, phi, flow)
    assert mon0["n_term3_active"] > 0
    frozen = (up0.to(torch.int64), torch.zeros(dm.n_tets, dtype=torch.int8, device="cuda"))
    Rf0 = ev.evaluate(phi, flow, jacobian=True, frozen=frozen).clone()
    Rr0 = ev.evaluate(phi, flow, jacobian=False).clone()
    # the residual-only gather sums in the row gather's order
    assert torch.equal(Rr0, R0)
    for shape in SHAPES:
        dm.set_tuning(*shape, assembly=0)
        R, J, up, rt, mon = _outputs(ev, phi, flow)
        assert torch.equal(R, R0), shape
        assert (J != J0).nnz == 0 and J.nnz == J0.nnz, shape
        assert torch.equal(up, up0) and torch.equal(rt, rt0)
        assert mon == mon0
        assert torch.equal(ev.evaluate(phi, flow, jacobian=True, frozen=frozen), Rf0)
        assert torch.equal(ev.evaluate(phi, flow, jacobian=False), Rr0)
    # the tiled form at each tile size: its own fixed order, the same
    # discrete decisions, the same values to rounding
    for T, stretch in ((128, 1), (256, 1), (256, 4)):
        dm.set_tuning(assembly=1, tile_elems=T, tile_stretch=stretch)
        R, J, up, rt, mon = _outputs(ev, phi, flow)
        assert torch.equal(up, up0) and torch.equal(rt, rt0) and mon == mon0, T
        assert rel_err(R.cpu().numpy(), R0.cpu().numpy()) < 1e-13, T
        assert J.nnz == J0.nnz and sparse_rel_err(J, J0) < 1e-13, T
        R2, J2, _, _, _ = _outputs(ev, phi, flow)
        assert torch.equal(R, R2) and (J != J2).nnz == 0
        assert torch.equal(ev.evaluate(phi, flow, jacobian=False), R)
        Rf = ev.evaluate(phi, flow, jacobian=True, frozen=frozen)
        assert rel_err(Rf.cpu().numpy(), Rf0.cpu().numpy()) < 1e-13
        info = dm.tile_info(T)
        assert info["tile_elems"] == T and info["tile_stretch"] == stretch
        assert info["n_tiles"] == -(-dm.n_tets // T)
        assert info["n_combined_nodes"] <= dm.n_nodes and info["n_combined_slots"] <= dm.nnz


def test_autotune_installs_a_listed_shape_and_keeps_parity():
    import torch
    from oracle import oracle as O
    from up3d_b200.solve.fused import FlowParams
    mesh, phi_h, dm, ev, phi = _setup()
    flow = FlowParams(m_inf=0.8)
    R0 = ev.evaluate(phi, flow, jacobian=True).clone()
    J0 = ev.jacobian().to_scipy()
    t = dm.autotune(phi, flow, reps=3)
    assert t == dm.tuning()
    assert (t["elem_persistent"], t["elem_threads_per_sm"]) in {(0, 512), (1, 512), (1, 640), (0, 768), (1, 768)}
    assert t["row_lanes"] in (4, 8, 16, 32) and t["row_plan8"] in (0, 1)
    assert t["assembly"] in (0, 1) and t["tile_elems"] in (128, 256) and t["tile_stretch"] in (1, 2, 4)
    assert t["elem_us"] > 0 and (t["row_us"] > 0 or t["assembly"] == 1)
    R = ev.evaluate(phi, flow, jacobian=True).clone()
    if t["assembly"] == 0:
        assert torch.equal(R, R0)
        assert (ev.jacobian().to_scipy() != J0).nnz == 0
    else:
        assert rel_err(R.cpu().numpy(), R0.cpu().numpy()) < 1e-13
    ref = O.chain(O.PicardOperator(mesh.nodes, mesh.elements),
                  O.UpwindOperator(mesh.nodes, mesh.elements), phi_h, 0.8)
    assert rel_err(R.cpu().numpy(), ref["R"]) < 1e-12


def test_bad_shapes_are_refused():
    _, _, dm, _, _ = _setup()
    for bad in [(2, 512, 8), (-1, 512, 8), (0, 256, 8), (0, 1024, 8), (0, 512, 2), (0, 512, 12), (0, 512, 64),
                (0, 512, 8, 2), (0, 512, 8, -1), (0, 512, 8, 0, 2), (0, 512, 8, 0, 1, 64), (0, 512, 8, 0, 1, 512),
                (0, 512, 8, 0, 1, 256, 3)]:
        with pytest.raises(ValueError):
            dm.set_tuning(*bad)
    assert dm.tuning()["row_lanes"] == 8


@pytest.mark.parametrize("ordering", ["morton", "hilbert"])
def test_renumbered_mesh_matches_the_oracle(ordering):
    """A renumbered mesh gives the oracle's results on the original
    numbering, permuted: upstream elements exactly, R and J within the
    parity tolerance (only the per-node summation order changes)."""
    import torch
    from oracle import oracle as O
    from up3d_b200.mesh.device import DeviceMesh
    from up3d_b200.mesh.kuhn import bump_channel, pocket_state
    from up3d_b200.mesh.order import renumber
    from up3d_b200.solve.fused import FlowParams, ResidualJacobian
    mesh = bump_channel(16, 6, 5, amplitude=0.08, seed=4)
    phi = pocket_state(mesh, "shockpoint")
    r = renumber(mesh.nodes, mesh.elements, ordering)
    dm = DeviceMesh(r.nodes, r.elements)
    ev = ResidualJacobian(dm)
    R = ev.evaluate(torch.from_numpy(r.nodal(phi)).cuda(), FlowParams(m_inf=0.8), jacobian=True)
    R = r.nodal_back(R.cpu().numpy())
    J = ev.jacobian().to_scipy()[r.node_inv][:, r.node_inv]
    up = r.element_ids_back(r.elemental_back(ev.upstream.cpu().numpy()))
    ref = O.chain(O.PicardOperator(mesh.nodes, mesh.elements),
                  O.UpwindOperator(mesh.nodes, mesh.elements), phi, 0.8)
    assert ref["n_term3_active"] > 0
    assert np.array_equal(up, ref["upstream"])
    assert rel_err(R, ref["R"]) < 1e-12
    D = (J - ref["J"]).tocoo()
    assert (np.abs(D.data).max() if D.nnz else 0.0) / np.abs(ref["J"].data).max() < 1e-12
