"""The Term-3 symbolic cache: a pocket state evaluated repeatedly (the
pattern recorded at its second evaluation, values only from the third on)
gives the same bits every time and matches the oracle; a different state
rebuilds the pattern and still matches; the frozen finish (fixed upstream
and branches) is served by the cache as well."""

import numpy as np
import pytest

from conftest import has_cuda, sparse_rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]


def test_repeated_pattern_is_served_values_only():
    import torch
    from oracle import oracle as O
    from up3d_b200.mesh.device import DeviceMesh
    from up3d_b200.mesh.kuhn import bump_channel, pocket_state
    from up3d_b200.solve.fused import FlowParams, ResidualJacobian
    mesh = bump_channel(20, 6, 5, amplitude=0.08, seed=5)
    dm = DeviceMesh(mesh.nodes, mesh.elements)
    ev = ResidualJacobian(dm)
    flow = FlowParams(m_inf=0.8)
    op, upw = O.PicardOperator(mesh.nodes, mesh.elements), O.UpwindOperator(mesh.nodes, mesh.elements)

    def run(fam, frozen=None):
        ev.evaluate(torch.from_numpy(pocket_state(mesh, fam)).cuda(), flow, frozen=frozen)
        return ev.R.clone(), ev.jacobian().to_scipy()

    h0 = dm.term3_cache_hits()
    outs = [run("mixed") for _ in range(4)]
    assert dm.term3_cache_hits() == h0 + 2
    for R, J in outs[1:]:
        assert torch.equal(R, outs[0][0])
        assert np.array_equal(J.indptr, outs[0][1].indptr) and np.array_equal(J.indices, outs[0][1].indices)
        assert np.array_equal(J.data, outs[0][1].data)
    ref = O.chain(op, upw, pocket_state(mesh, "mixed"), 0.8)
    assert ref["n_term3_active"] > 0
    assert sparse_rel_err(outs[-1][1], ref["J"]) < 1e-12
    # another pattern, then back: rebuilt, still the oracle's
    h1 = dm.term3_cache_hits()
    _, Ja = run("accelerating")
    refa = O.chain(op, upw, pocket_state(mesh, "accelerating"), 0.8)
    assert sparse_rel_err(Ja, refa["J"]) < 1e-12
    _, Jm = run("mixed")
    assert dm.term3_cache_hits() == h1
    assert np.array_equal(Jm.data, outs[0][1].data)
    # the frozen finish: fixed (upstream, branch), repeated
    up = ev.upstream.to(torch.int64).clone()
    ws_br = torch.ones(dm.n_tets, dtype=torch.int8, device="cuda")
    fz = [run("mixed", frozen=(up, ws_br)) for _ in range(3)]
    assert dm.term3_cache_hits() >= h1 + 1
    assert np.array_equal(fz[2][1].data, fz[0][1].data) and torch.equal(fz[2][0], fz[0][0])
