"""element_velocity_q2 on the B200 (pyfp3d/kernels/gradient.py:33-64)."""

from __future__ import annotations

import numpy as np

from .. import _lib as L


def element_velocity_q2(elements, B, phi, grad_out, q2_out) -> None:
    """grad(phi)_e = sum_i phi_i B_e[i, :] and q^2_e = |grad(phi)_e|^2, into
    the preallocated outputs (numpy arrays or CUDA tensors)."""
    t = L.torch()
    d_el = L.to_device(elements, t.int32)
    d_B = L.to_device(B, t.float64)
    d_phi = L.to_device(phi, t.float64)
    E = d_el.shape[0]
    if L.is_torch(grad_out) and grad_out.is_cuda and grad_out.is_contiguous():
        g, q = grad_out, q2_out
    else:
        g = t.empty((E, 3), dtype=t.float64, device="cuda")
        q = t.empty(E, dtype=t.float64, device="cuda")
    L.call("up3d_element_velocity_q2", d_el.data_ptr(), d_B.data_ptr(), d_phi.data_ptr(), E,
           g.data_ptr(), q.data_ptr(), L.stream_ptr())
    if g is not grad_out:
        if L.is_torch(grad_out):
            grad_out.copy_(g)
            q2_out.copy_(q)
        else:
            np.copyto(grad_out, g.cpu().numpy())
            np.copyto(q2_out, q.cpu().numpy())
