"""The library's device block cache (up3d_pool_stats / up3d_pool_release):
a mesh, evaluation and AMG hierarchy built a second time are served from
the blocks the first one freed, with the same results; a release empties
the cache; UP3D_POOL_CACHE_MB=0 turns caching off."""

import gc
import os
import subprocess
import sys
from pathlib import Path

import pytest

from conftest import has_cuda

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_cuda(), reason="needs a CUDA device")]

REPO = Path(__file__).resolve().parents[1]


def _setup_and_solve(mesh, phi_h):
    import torch
    from up3d_b200.mesh.device import DeviceMesh
    from up3d_b200.solve.fused import FlowParams, ResidualJacobian
    from up3d_b200.solve.linear import build_amg_preconditioner
    dm = DeviceMesh(mesh.nodes, mesh.elements)
    ev = ResidualJacobian(dm)
    R = ev.evaluate(torch.from_numpy(phi_h).cuda(), FlowParams(m_inf=0.8), jacobian=True).clone()
    J = ev.jacobian().to_scipy()
    _, M = build_amg_preconditioner(J)
    z = M.matvec(R)
    torch.cuda.synchronize()
    return R.cpu(), J, z.cpu()


def test_repeated_setup_is_served_from_the_cache():
    from up3d_b200 import _lib as L
    from up3d_b200.mesh.kuhn import bump_channel, pocket_state
    mesh = bump_channel(24, 8, 6, amplitude=0.08, seed=1)
    phi_h = pocket_state(mesh, "mixed")
    R0, J0, z0 = _setup_and_solve(mesh, phi_h)
    gc.collect()
    s0 = L.pool_stats()
    assert s0["cached_bytes"] > 0
    R1, J1, z1 = _setup_and_solve(mesh, phi_h)
    gc.collect()
    s1 = L.pool_stats()
    hits, misses = s1["hits"] - s0["hits"], s1["misses"] - s0["misses"]
    assert hits > 0 and misses <= hits // 4, (hits, misses)
    # the same bits from reused blocks
    assert (R0 == R1).all() and (J0 != J1).nnz == 0 and (z0 == z1).all()
    released = L.pool_release()
    s2 = L.pool_stats()
    assert released == s1["cached_bytes"] and s2["cached_bytes"] == 0
    assert s2["live_bytes"] == s1["live_bytes"]


def test_cache_off_by_environment():
    code = (
        "import gc, torch\n"
        "from up3d_b200 import _lib as L\n"
        "from up3d_b200.mesh.device import DeviceMesh\n"
        "from up3d_b200.mesh.kuhn import bump_channel\n"
        "m = bump_channel(8, 4, 3, amplitude=0.05, seed=0)\n"
        "for _ in range(2):\n"
        "    dm = DeviceMesh(m.nodes, m.elements)\n"
        "    del dm\n"
        "    gc.collect()\n"
        "s = L.pool_stats()\n"
        "assert s['cached_bytes'] == 0 and s['hits'] == 0 and s['misses'] > 0, s\n"
        "print('ok')\n")
    env = dict(os.environ, UP3D_POOL_CACHE_MB="0")
    out = subprocess.run([sys.executable, "-c", code], cwd=REPO, env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip().endswith("ok")
