"""Cut-element assembly of the level-set wake, with the reference's
signatures (pyfp3d/kernels/cut_assembly.py:47-556).

* newton_terms23_side_coo: one side's Newton Terms 2 and 3 as COO on the
  extended DOFs, on the device (up3d_terms23_side_coo); the level-set path
  runs the walk flux once per side on a face graph restricted to that
  side's elements (``UpwindOperator.face_neighbors = fn``).  Arrays in,
  same kind out.
* the extended-matrix corrections (redirection, weld rows, two-sided mass
  conservation, wake least squares) as host COO over the cut elements, in
  the reference's triplet order; wake.multivalued adds them to the device
  P1 matrix.
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


# ------------------------------------------------ cut-element corrections
#
# The extended (multivalued) matrix of the level-set path is the ordinary
# P1 matrix plus corrections that involve the cut elements only
# (pyfp3d/kernels/cut_assembly.py:47-238, :539-556).  They are formed here
# on the host over those few elements, as COO triplets in the reference's
# order; wake.multivalued folds them into a device CSR whose pattern is
# planned once.

def _host(x, dtype=None):
    if L.is_torch(x):
        x = x.detach().cpu().numpy()
    return np.asarray(x) if dtype is None else np.asarray(x, dtype=dtype)


def cut_element_stiffness(B_cut, V_cut, rho_cut):
    """(n, 4, 4) element matrices rho_e V_e (B_a . B_b)."""
    B = _host(B_cut, np.float64)
    w = _host(V_cut, np.float64) * _host(rho_cut, np.float64)
    return np.einsum("e,ead,ebd->eab", w, B, B)


def _geometry(op, ids):
    """B and V of the listed elements (host)."""
    if hasattr(op, "cut_geometry"):
        return op.cut_geometry(ids)
    return _host(op.B)[ids], _host(op.V)[ids]


def _weights(rho, ids):
    return np.ones(len(ids)) if rho is None else _host(rho, np.float64)[ids]


def multivalued_redirection_coo(op, cm, rho_tilde=None):
    """COO moving each cut element's opposite-side entries K[a, b] from the
    column main(b) to aux(b): -K at (main(a), main(b)), +K at (main(a),
    aux(b)) -- the single-valued matrix plus these is the multivalued one
    (kernels/cut_assembly.py:56-103)."""
    cut = np.asarray(cm.cut_elems, dtype=np.int64)
    if len(cut) == 0:
        z = np.empty(0, dtype=np.int64)
        return z, z, np.empty(0)
    conn = _host(op.elements, np.int64)[cut]
    B, V = _geometry(op, cut)
    K = cut_element_stiffness(B, V, _weights(rho_tilde, cut))
    side = cm.node_side[conn]
    aux = cm.ext_dof_of_node[conn]
    e, a, b = np.nonzero(side[:, :, None] != side[:, None, :])
    row = conn[e, a]
    k = K[e, a, b]
    return (np.concatenate([row, row]), np.concatenate([conn[e, b], aux[e, b]]), np.concatenate([-k, k]))


def nonte_aux_rows(cm):
    """Aux DOFs of the cut nodes that are not TE nodes: the rows the wake
    least-squares condition replaces (kernels/cut_assembly.py:106-116)."""
    te = np.zeros(cm.n_main, dtype=bool)
    te[cm.te_nodes] = True
    cut_nodes = np.flatnonzero(cm.ext_dof_of_node >= 0)
    return cm.ext_dof_of_node[cut_nodes[~te[cut_nodes]]].astype(np.int64)


def special_elements(cm, n_tets):
    """(plain, is_special): elements assembled single-valued on the main
    DOFs, and the mask of cut + below-TE-fan elements."""
    special = np.zeros(n_tets, dtype=bool)
    special[cm.cut_elems] = True
    special[cm.te_lower_elems] = True
    return np.flatnonzero(~special), special


def mass_conservation_coo(op, cm, rho_upper=None, rho_lower=None, elements="all"):
    """The multivalued mass-conservation matrix as COO
    (kernels/cut_assembly.py:119-182): plain elements once on their main
    DOFs with their own side's density, cut elements twice (upper and lower
    DOF vectors, each side's density), below-TE-fan elements with the TE
    node's aux DOF and the lower density.  elements="special" gives the cut
    and fan parts alone (the plain part is the device P1 assembly)."""
    el = _host(op.elements, np.int64)
    E = len(el)
    if rho_upper is None and rho_lower is None:
        ru = rl = np.ones(E)
    else:
        ru, rl = _host(rho_upper, np.float64), _host(rho_lower, np.float64)
    te = np.zeros(cm.n_main, dtype=bool)
    te[cm.te_nodes] = True
    tel = np.asarray(cm.te_lower_elems, dtype=np.int64)
    tel_dof = np.where(te[el[tel]], cm.ext_dof_of_node[el[tel]], el[tel])
    parts = []
    if elements == "all":
        plain, _ = special_elements(cm, E)
        plus = cm.node_side[el[plain]].max(axis=1) == 1
        parts.append((plain, el[plain], np.where(plus, ru[plain], rl[plain])))
    cut = np.asarray(cm.cut_elems, dtype=np.int64)
    parts += [(cut, cm.dofs_upper, ru[cut]), (cut, cm.dofs_lower, rl[cut]), (tel, tel_dof, rl[tel])]
    rows, cols, data = [], [], []
    for ids, dof, w in parts:
        if len(ids) == 0:
            continue
        B, V = _geometry(op, ids)
        K = cut_element_stiffness(B, V, w)
        rows.append(np.repeat(dof, 4, axis=1).ravel())
        cols.append(np.tile(dof, (1, 4)).ravel())
        data.append(K.ravel())
    if not rows:
        z = np.empty(0, dtype=np.int64)
        return z, z, np.empty(0)
    return np.concatenate(rows).astype(np.int64), np.concatenate(cols).astype(np.int64), np.concatenate(data)


def wake_ls_coo(op, cm, wake_normal, u_hat):
    """Wake least-squares rows (kernels/cut_assembly.py:185-265): per cut
    element, P_ac = (n.B_a)(n.B_c) + (u.B_a)(u.B_c) times V_e, on the aux
    row of each non-TE node a, +V P_ac on the upper DOF of c and -V P_ac on
    the lower DOF of c."""
    cut = np.asarray(cm.cut_elems, dtype=np.int64)
    if len(cut) == 0:
        z = np.empty(0, dtype=np.int64)
        return z, z, np.empty(0)
    conn = _host(op.elements, np.int64)[cut]
    B, V = _geometry(op, cut)
    n = np.asarray(wake_normal, dtype=np.float64)
    u = np.asarray(u_hat, dtype=np.float64)
    u = u / np.linalg.norm(u)
    bn = np.einsum("ead,ed->ea", B, n)
    bu = np.einsum("ead,d->ea", B, u)
    VP = V[:, None, None] * (bn[:, :, None] * bn[:, None, :] + bu[:, :, None] * bu[:, None, :])
    te = np.zeros(cm.n_main, dtype=bool)
    te[cm.te_nodes] = True
    ok = ~te[conn]
    e, a, c = np.nonzero(ok[:, :, None] & np.ones((1, 1, 4), dtype=bool))
    k = VP[e, a, c]
    row = cm.ext_dof_of_node[conn][e, a]
    up = np.asarray(cm.dofs_upper, dtype=np.int64)
    lo = np.asarray(cm.dofs_lower, dtype=np.int64)
    return np.concatenate([row, row]), np.concatenate([up[e, c], lo[e, c]]), np.concatenate([k, -k])


def continuity_closure_coo(cm):
    """The weld rows aux_k - main_j = 0 of every cut node j
    (kernels/cut_assembly.py:539-556)."""
    nodes = np.flatnonzero(cm.ext_dof_of_node >= 0).astype(np.int64)
    aux = cm.ext_dof_of_node[nodes]
    one = np.ones(len(aux))
    return np.concatenate([aux, aux]), np.concatenate([aux, nodes]), np.concatenate([one, -one])
