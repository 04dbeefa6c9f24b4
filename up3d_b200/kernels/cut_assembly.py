"""Per-side Newton Terms 2 and 3 of the level-set (cut-element) assembly on
the B200, with the reference's signature (pyfp3d/kernels/cut_assembly.py:
401-488).

The level-set path runs the walk flux once per side on a face graph
restricted to that side's elements; ``UpwindOperator.face_neighbors = fn``
installs such a masked graph on the device.  This module adds the side's
density-sensitivity blocks as COO triplets on the extended DOFs
(``up3d_terms23_side_coo``).  Arrays in, same kind out.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .. import _lib as L


def newton_terms23_side_coo(op, side, u_inf: float = 1.0):
    """(rows, cols, data) of one side's Terms 2 + 3 (module docstring).
    `op` is this package's PicardOperator (its mesh holds B and V); `side`
    the reference's side record: keep, dofvec, readvec (optional), grad,
    grad_row (optional), lim_mask, s_e, s_u, upstream."""
    t = L.require_cuda()
    mesh = op._mesh
    E = mesh.n_tets
    dev = L.is_torch(side["grad"])
    keep = L.to_device(side["keep"], t.uint8)
    dof = L.to_device(side["dofvec"], t.int64)
    read = side.get("readvec")
    read = L.to_device(read, t.int64) if read is not None else None
    grad = L.to_device(side["grad"], t.float64)
    grow = side.get("grad_row")
    grow = L.to_device(grow, t.float64) if grow is not None else None
    lim = L.to_device(side["lim_mask"], t.float64)
    s_e = L.to_device(side["s_e"], t.float64)
    s_u = L.to_device(side["s_u"], t.float64)
    up = L.to_device(side["upstream"], t.int64)
    for name, a, n in (("keep", keep, E), ("dofvec", dof, 4 * E), ("grad", grad, 3 * E),
                       ("lim_mask", lim, E), ("s_e", s_e, E), ("s_u", s_u, E), ("upstream", up, E)):
        if a.numel() != n:
            raise ValueError(f"{name} has {a.numel()} entries, expected {n}")
    count = ctypes.c_int64()
    args = [mesh.handle, keep.data_ptr(), dof.data_ptr(), L.ptr(read), grad.data_ptr(), L.ptr(grow),
            lim.data_ptr(), s_e.data_ptr(), s_u.data_ptr(), up.data_ptr(), float(u_inf)]
    L.call("up3d_terms23_side_coo", *args, None, None, None, 0, ctypes.byref(count), L.stream_ptr())
    n = count.value
    rows = t.empty(max(n, 1), dtype=t.int64, device="cuda")
    cols = t.empty(max(n, 1), dtype=t.int64, device="cuda")
    data = t.empty(max(n, 1), dtype=t.float64, device="cuda")
    L.call("up3d_terms23_side_coo", *args, rows.data_ptr(), cols.data_ptr(), data.data_ptr(), n,
           ctypes.byref(count), L.stream_ptr())
    rows, cols, data = rows[:n], cols[:n], data[:n]
    if dev:
        return rows, cols, data
    return rows.cpu().numpy(), cols.cpu().numpy(), data.cpu().numpy()
