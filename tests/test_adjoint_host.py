"""Host-side pieces of the adjoint and batched forms (no GPU): the shape
parametrisation, the lower-wall faces, the CSR transpose and the batched
mesh union."""

import numpy as np
import pytest


def test_bump_shape_reproduces_bump_channel_and_its_derivative():
    from up3d_b200.adjoint import BumpShape
    from up3d_b200.mesh.kuhn import bump_channel
    shape = BumpShape(12, 5, 4, amplitude=0.06, seed=3)
    ref = bump_channel(12, 5, 4, amplitude=0.06, seed=3)
    assert np.array_equal(shape.nodes(), ref.nodes)
    assert np.array_equal(shape.elements, ref.elements)
    assert shape.n_params == 16
    # z is affine in p: the derivative is exact for any step
    rng = np.random.default_rng(0)
    p = rng.standard_normal(shape.n_params) * 1e-3
    dz = shape.nodes(p)[:, 2] - shape.nodes()[:, 2]
    assert np.allclose(dz, shape.dz_dp() @ p, rtol=0, atol=1e-15)
    # x, y never move; the upper wall (z = 1) does not move
    assert np.array_equal(shape.nodes(p)[:, :2], shape.nodes()[:, :2])
    top = np.isclose(shape.box[:, 2], 1.0)
    assert np.array_equal(shape.nodes(p)[top, 2], shape.nodes()[top, 2])


def test_lower_wall_faces():
    from up3d_b200.adjoint import lower_wall_faces
    from up3d_b200.mesh.kuhn import bump_channel
    nx, ny, nz = 7, 4, 3
    m = bump_channel(nx, ny, nz, amplitude=0.05, seed=1)
    faces = lower_wall_faces(m.elements, m.shape)
    assert len(faces) == 2 * nx * ny            # two triangles per wall quad
    assert np.all(faces[:, 1:] % (nz + 1) == 0)  # all on k = 0
    for e, a, b, c in faces:                     # the three nodes belong to the element
        assert {a, b, c} <= set(m.elements[e].tolist())
    assert len({tuple(sorted(f[1:])) for f in faces}) == len(faces)


def test_transpose_csr_matches_scipy():
    import scipy.sparse as sp
    import torch
    from up3d_b200.adjoint import transpose_csr
    from up3d_b200.mesh.device import DeviceCSR
    A = sp.random(40, 30, density=0.2, random_state=np.random.default_rng(4), format="csr")
    A.sort_indices()
    d = DeviceCSR(torch.from_numpy(A.indptr.astype(np.int32)), torch.from_numpy(A.indices.astype(np.int32)),
                  torch.from_numpy(A.data), A.shape)
    T = transpose_csr(d)
    ref = A.T.tocsr()
    ref.sort_indices()
    assert T.shape == (30, 40)
    assert np.array_equal(T.indptr.numpy(), ref.indptr)
    assert np.array_equal(T.indices.numpy(), ref.indices)
    assert np.array_equal(T.data.numpy(), ref.data)
