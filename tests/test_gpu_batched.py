"""Several channel cases in one mesh: the batched residual/Jacobian equals
the per-case evaluations bit for bit, and the lockstep Newton reaches the
per-case plain solves' potentials."""

import numpy as np
import pytest

from conftest import has_cuda

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]


def _cases():
    from up3d_b200.mesh.kuhn import bump_channel
    return [bump_channel(10, 4, 3, amplitude=0.08, seed=1), bump_channel(14, 5, 4, amplitude=0.03, seed=2),
            bump_channel(8, 3, 3, amplitude=0.05, seed=3)]


def test_batched_evaluation_equals_per_case_bitwise():
    import torch
    from up3d_b200.mesh.kuhn import pocket_state
    from up3d_b200.solve.batched import BatchedChannels
    from up3d_b200.solve.fused import FlowParams
    from up3d_b200.solve.newton import ChannelWorkspace
    meshes = _cases()
    machs = [0.8, 0.6, 0.85]
    fams = ["mixed", "accelerating", "shockpoint"]
    batch = BatchedChannels(meshes)
    phis = [pocket_state(m, f) for m, f in zip(meshes, fams)]
    phi = torch.from_numpy(np.concatenate(phis)).cuda()
    R = batch.evaluate(phi, machs, jacobian=True).clone()
    Jb = batch.ws.ev.jacobian().to_scipy()
    for c, (m, p, M) in enumerate(zip(meshes, phis, machs)):
        ws = ChannelWorkspace(m.nodes, m.elements, m.dirichlet_nodes)
        Rc = ws.ev.evaluate(torch.from_numpy(p).cuda(), FlowParams(m_inf=M), jacobian=True).clone()
        a, b = batch.node_off[c], batch.node_off[c + 1]
        assert torch.equal(R[a:b], Rc)
        Jc = ws.ev.jacobian().to_scipy()
        blk = Jb[a:b][:, a:b].tocsr()
        assert (blk != Jc).nnz == 0
    assert (Jb[batch.node_off[0]:batch.node_off[1]][:, batch.node_off[1]:]).nnz == 0


def test_case_index_out_of_range_raises():
    import torch
    from up3d_b200.solve.batched import BatchedChannels
    batch = BatchedChannels(_cases()[:2])
    batch.case_of_elem[0] = 5
    with pytest.raises(ValueError, match="case index"):
        batch.evaluate(batch.ws.freestream.clone(), [0.5, 0.5])


def test_batched_newton_matches_plain_solves():
    from up3d_b200.solve.batched import BatchedChannels, solve_newton_batched
    from up3d_b200.solve.newton import ChannelWorkspace, solve_newton_transonic
    meshes = _cases()
    machs = [0.6, 0.5, 0.7]
    batch = BatchedChannels(meshes)
    res = solve_newton_batched(batch, machs)
    assert res["converged"].all(), res
    phi = res["phi"].cpu().numpy()
    for c, (m, M) in enumerate(zip(meshes, machs)):
        ws = ChannelWorkspace(m.nodes, m.elements, m.dirichlet_nodes)
        r = solve_newton_transonic(ws, M, m_start=min(0.70, M))
        assert r["converged"]
        ref = r["phi"].cpu().numpy()
        a, b = batch.node_off[c], batch.node_off[c + 1]
        assert np.abs(phi[a:b] - ref).max() < 1e-8


def test_graph_replayed_trial_merits_match_direct_evaluation():
    import torch
    from up3d_b200.mesh.kuhn import pocket_state
    from up3d_b200.solve.batched import BatchedChannels
    meshes = _cases()
    machs = [0.8, 0.6, 0.85]
    batch = BatchedChannels(meshes)
    mask_b = batch.ws.mask.bool()
    phi = torch.from_numpy(np.concatenate([pocket_state(m, f) for m, f in
                                           zip(meshes, ["mixed", "accelerating", "shockpoint"])])).cuda()
    dphi = torch.from_numpy(np.random.default_rng(5).standard_normal(len(phi)) * 1e-3).cuda()
    dphi = dphi.masked_fill(mask_b, 0.0)
    batch.evaluate(phi, machs, jacobian=True)   # uploads the flows, as the Newton loop does
    for lam in ([1.0, 0.5, 0.25], [0.0, 1.0, 0.125], [0.5, 0.5, 0.5]):
        m_graph = batch.trial_merits(phi, dphi, np.array(lam), mask_b)
        lam_node = torch.tensor(lam, dtype=torch.float64, device="cuda")[batch.case_of_node]
        R = batch.evaluate(phi + lam_node * dphi, machs, jacobian=False)
        m_direct = batch.per_case(R.masked_fill(mask_b, 0.0), "sumsq").cpu().numpy()
        assert np.allclose(m_graph, m_direct, rtol=1e-12, atol=0)
    # machs=None without a table of this many cases on the mesh is refused
    other = BatchedChannels(meshes[:2])
    with pytest.raises(ValueError, match="flow table"):
        other.evaluate(other.ws.freestream.clone(), None)


@pytest.mark.parametrize("ordering", ["morton", "hilbert"])
def test_renumbered_batch_matches_per_case_evaluations(ordering):
    import torch
    from up3d_b200.mesh.kuhn import pocket_state
    from up3d_b200.solve.batched import BatchedChannels
    from up3d_b200.solve.fused import FlowParams
    from up3d_b200.solve.newton import ChannelWorkspace
    meshes = _cases()
    machs = [0.8, 0.6, 0.85]
    phis = [pocket_state(m, f) for m, f in zip(meshes, ["mixed", "accelerating", "shockpoint"])]
    batch = BatchedChannels(meshes, ordering=ordering)
    phi = batch.union_phi(phis)
    R = batch.evaluate(phi, machs, jacobian=True).clone()
    for c, (m, p, M) in enumerate(zip(meshes, phis, machs)):
        assert torch.equal(batch.case_phi(phi, c).cpu(), torch.from_numpy(p))
        ws = ChannelWorkspace(m.nodes, m.elements, m.dirichlet_nodes)
        Rc = ws.ev.evaluate(torch.from_numpy(p).cuda(), FlowParams(m_inf=M), jacobian=True)
        Rb = batch.case_phi(R, c)
        scale = Rc.abs().max()
        assert float((Rb - Rc).abs().max() / scale) < 1e-12


def test_tuned_batch_picks_an_ordering_and_converges():
    from up3d_b200.solve.batched import BatchedChannels, solve_newton_batched
    meshes = _cases()[:2]
    machs = [0.6, 0.5]
    batch = BatchedChannels.tuned(meshes, machs, reps=3)
    rep = batch.tuning_report
    assert rep["ordering"] == batch.ordering
    assert set(rep["candidates"]) == {"given", "morton", "hilbert"}
    assert all(v["ms"] > 0 for v in rep["candidates"].values())
    res = solve_newton_batched(batch, machs)
    assert res["converged"].all()


def test_compacted_batch_matches_plain_solves():
    """Compaction onto the unfinished cases (as soon as one case has
    finished) carries their potentials and frozen selections over: the
    same converged potentials as the plain solves."""
    from up3d_b200.solve.batched import BatchedChannels, solve_newton_batched
    from up3d_b200.solve.newton import ChannelWorkspace, solve_newton_transonic
    meshes = _cases()
    machs = [0.5, 0.5, 0.75]        # the third case alone goes on to a second Mach level
    batch = BatchedChannels(meshes)
    res = solve_newton_batched(batch, machs, compact_fraction=1.0)
    assert res["converged"].all(), res
    assert res["n_compactions"] >= 1
    phi = res["phi"].cpu().numpy()
    for c, (m, M) in enumerate(zip(meshes, machs)):
        ws = ChannelWorkspace(m.nodes, m.elements, m.dirichlet_nodes)
        r = solve_newton_transonic(ws, M, m_start=min(0.70, M))
        a, b = batch.node_off[c], batch.node_off[c + 1]
        assert np.abs(phi[a:b] - r["phi"].cpu().numpy()).max() < 1e-8


def test_case_set_batches_the_small_cases_and_runs_the_rest_alone():
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.solve.batched import CaseSet
    from up3d_b200.solve.newton import ChannelWorkspace, solve_newton_transonic
    meshes = _cases() + [bump_channel(24, 8, 6, amplitude=0.04, seed=4)]
    machs = [0.6, 0.5, 0.7, 0.65]
    cs = CaseSet(meshes, machs, batch_below=1000)
    assert sorted(cs.small.tolist()) == [0, 2] and sorted(cs.large.tolist()) == [1, 3]
    res = cs.solve()
    assert res["converged"].all() and res["n_batched"] == 2 and res["n_plain"] == 2
    assert np.all(np.isfinite(res["case_s"])) and res["time_s"] >= np.nanmax(res["case_s"]) - 1e-9
    for c, (m, M) in enumerate(zip(meshes, machs)):
        ws = ChannelWorkspace(m.nodes, m.elements, m.dirichlet_nodes)
        r = solve_newton_transonic(ws, M, m_start=min(0.70, M))
        assert np.abs(res["phi"][c].cpu().numpy() - r["phi"].cpu().numpy()).max() < 1e-8
    # one small case alone is not batched
    one = CaseSet(meshes[:2], machs[:2], batch_below=1000)
    assert one.batch is None and len(one.large) == 2
