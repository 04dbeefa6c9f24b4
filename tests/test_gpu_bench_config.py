"""Parity at the benchmark's own configuration: the transonic bump channel
of 200 x 60 x 50 hexes (3.6 M tets, bump 0.08, M_inf 0.85), the residual,
the upwinded density, the upstream map, the live branch of every element
and the merged Newton Jacobian (Terms 1-3) of the fused evaluation against
the oracle's composition of the reference kernels (the chain of
pyfp3d/solve/newton.py:345-372 and :430-457 without a wake), at the five
seeded states the benchmark times and at the three supersonic-pocket
families (Term 3 active).  Floating-point outputs within 1e-12 of the
oracle's largest magnitude (the Jacobian over the union pattern), integer
outputs exact.  Both assembly forms (tiled and two-pass) are checked."""

import numpy as np
import pytest

from conftest import has_cuda, rel_err, sparse_rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]

SHAPE = (200, 60, 50)
M_INF = 0.85
STATES = [("seed", k) for k in range(5)] + [("pocket", f) for f in ("accelerating", "shockpoint", "mixed")]


@pytest.fixture(scope="module")
def c2():
    import torch
    from oracle import oracle as O
    from up3d_b200.mesh.device import DeviceMesh
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.solve.fused import ResidualJacobian
    mesh = bump_channel(*SHAPE, amplitude=0.08, seed=0)
    dm = DeviceMesh(mesh.nodes, mesh.elements)
    ev = ResidualJacobian(dm)
    op = O.PicardOperator(mesh.nodes, mesh.elements)
    upw = O.UpwindOperator(mesh.nodes, mesh.elements)
    case_of = torch.zeros(dm.n_tets, dtype=torch.int32, device="cuda")
    branch = torch.empty(dm.n_tets, dtype=torch.int8, device="cuda")
    return mesh, dm, ev, op, upw, case_of, branch


def _phi(mesh, kind, k):
    from up3d_b200.mesh.kuhn import pocket_state, seeded_state
    return seeded_state(mesh, k) if kind == "seed" else pocket_state(mesh, k)


def _device(c2, phi_h):
    """R, J, rho~, upstream and the live branch of one fused evaluation (the
    branch through the batched entry point with one case), and the
    residual-only R."""
    import torch
    from up3d_b200 import _lib as L
    from up3d_b200.solve.fused import FlowParams
    mesh, dm, ev, op, upw, case_of, branch = c2
    phi = torch.from_numpy(phi_h).cuda()
    flow = FlowParams(m_inf=M_INF)
    ev.evaluate(phi, flow, jacobian=True)
    R = ev.R.cpu().numpy()
    J = ev.jacobian().to_scipy()
    rt = ev.rho_tilde.cpu().numpy()
    up = ev.upstream.cpu().numpy()
    mon = ev.read_monitors()
    flows = (L.Flow * 1)()
    flows[0] = flow.c()
    R2 = torch.empty_like(ev.R)
    L.call("up3d_residual_jacobian_batched", dm.handle, phi.data_ptr(), 1, flows, case_of.data_ptr(), None, None,
           R2.data_ptr(), None, None, None, branch.data_ptr(), None, L.stream_ptr())
    return R, J, rt, up, branch.cpu().numpy(), mon, R2.cpu().numpy()


def _oracle(c2, phi_h):
    from oracle import oracle as O
    mesh, dm, ev, op, upw, case_of, branch = c2
    ref = O.chain(op, upw, phi_h, M_INF)
    _, br = upw.freeze_upwind_state(ref["grad"], ref["q2l"], ref["rho"], M_INF, O.UPWIND_C, O.M_CRIT)
    return ref, br


@pytest.mark.parametrize("assembly", [1, 0])
def test_bench_configuration_matches_the_oracle(c2, assembly):
    mesh, dm, ev, op, upw, case_of, branch = c2
    assert dm.n_tets == 3_600_000
    dm.set_tuning(assembly=assembly)
    n_pocket_active = 0
    for kind, k in STATES:
        phi_h = _phi(mesh, kind, k)
        R, J, rt, up, br, mon, R_res = _device(c2, phi_h)
        ref, br_ref = _oracle(c2, phi_h)
        tag = f"{kind} {k} assembly={assembly}"
        assert rel_err(R, ref["R"]) < 1e-12, tag
        assert rel_err(R_res, ref["R"]) < 1e-12, tag
        assert rel_err(rt, ref["rho_tilde"]) < 1e-12, tag
        assert np.array_equal(up, ref["upstream"]), tag
        assert np.array_equal(br, br_ref), tag
        assert mon["n_supersonic"] == ref["n_supersonic"], tag
        assert mon["n_floored"] == ref["n_floored"], tag
        assert mon["n_limited"] == ref["n_limited"], tag
        assert mon["n_term3_active"] == ref["n_term3_active"], tag
        assert J.shape == ref["J"].shape
        assert sparse_rel_err(J, ref["J"]) < 1e-12, tag
        if kind == "pocket":
            n_pocket_active += int(ref["n_term3_active"] > 0)
    assert n_pocket_active == 3
