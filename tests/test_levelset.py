"""The level-set wake's host side against the reference
(tests/golden/multivalued.npz, made by make_golden.py from
pyfp3d/wake/levelset.py, cut_elements.py, multivalued.py and
kernels/cut_assembly.py): the level set at the nodes and the sheet normals
bitwise, the cut census and extended-DOF numbering exactly, and the
extended matrices rebuilt from the oracle's P1 operator plus this package's
cut-element corrections within 1e-12."""

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN, sparse_rel_err


@pytest.fixture(scope="module")
def case():
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.wake.cut_elements import CutElementMap
    from up3d_b200.wake.levelset import WakeLevelSet
    g = np.load(GOLDEN / "multivalued.npz")
    mesh = bump_channel(16, 6, 5, amplitude=0.08, seed=3)
    ls = WakeLevelSet(g["te_points"], g["direction"])
    cm = CutElementMap(mesh.nodes, mesh.elements, ls)
    return g, mesh, ls, cm


def _csr(g, tag, n):
    return sp.csr_matrix((g[tag + "/data"], g[tag + "/indices"], g[tag + "/indptr"]), shape=(n, n))


def test_level_set_and_census_match_the_reference(case):
    g, mesh, ls, cm = case
    s, d, q = ls.evaluate(mesh.nodes)
    assert np.array_equal(s, g["s"]) and np.array_equal(d, g["d"]) and np.array_equal(q, g["q"])
    cen = mesh.nodes[mesh.elements[cm.cut_elems]].mean(axis=1)
    assert np.array_equal(ls.surface_normals(cen), g["normals_cut"])
    for k in ("node_side", "te_nodes", "cut_elems", "te_lower_elems", "beyond_tip_elems", "shifted_nodes",
              "ext_dof_of_node", "dofs_upper", "dofs_lower"):
        assert np.array_equal(getattr(cm, k), g[k]), k
    assert cm.n_total_dofs == int(g["n_total"])
    assert len(cm.cut_elems) > 100 and cm.n_ext_dofs > 50


def test_extended_matrices_from_the_cut_element_corrections(case):
    """P1 matrix (oracle) + redirection + weld rows = the reference's
    continuity matrix; plain part (oracle, plain elements weighted by their
    side's density) + two-sided cut copies + wake least squares = its
    wake_ls matrix."""
    from oracle import oracle as O
    from up3d_b200.kernels import cut_assembly as ca
    g, mesh, ls, cm = case
    op = O.PicardOperator(mesh.nodes, mesh.elements)
    n = cm.n_total_dofs
    nm = cm.n_main

    def embed(A):
        A = A.tocoo()
        return sp.csr_matrix((A.data, (A.row, A.col)), shape=(n, n))

    rho = g["rho_main"]
    for tag, w in (("A_laplace", None), ("A_continuity", rho)):
        r = ca.multivalued_redirection_coo(op, cm, w)
        c = ca.continuity_closure_coo(cm)
        corr = sp.csr_matrix((np.concatenate([r[2], c[2]]), (np.concatenate([r[0], c[0]]),
                                                              np.concatenate([r[1], c[1]]))), shape=(n, n))
        A = embed(op.assemble_matrix(w)) + corr
        assert sparse_rel_err(A, _csr(g, tag, n)) < 1e-12, tag
    ru, rl = g["rho_up"], g["rho_lo"]
    plain, special = ca.special_elements(cm, len(mesh.elements))
    plus = cm.node_side[mesh.elements].max(axis=1) == 1
    w = np.where(plus, ru, rl)
    w[special] = 0.0
    m = ca.mass_conservation_coo(op, cm, ru, rl, elements="special")
    drop = np.zeros(n, dtype=bool)
    drop[ca.nonte_aux_rows(cm)] = True
    keep = ~drop[m[0]]
    cen = mesh.nodes[mesh.elements[cm.cut_elems]].mean(axis=1)
    lsc = ca.wake_ls_coo(op, cm, ls.surface_normals(cen), ls.direction)
    corr = sp.csr_matrix((np.concatenate([m[2][keep], lsc[2]]),
                          (np.concatenate([m[0][keep], lsc[0]]), np.concatenate([m[1][keep], lsc[1]]))),
                         shape=(n, n))
    A = embed(op.assemble_matrix(w)) + corr
    assert sparse_rel_err(A, _csr(g, "A_wake_ls", n)) < 1e-12
    # the full two-sided mass conservation (plain elements included) agrees
    full = ca.mass_conservation_coo(op, cm, ru, rl)
    Mf = sp.csr_matrix((full[2], (full[0], full[1])), shape=(n, n))
    Ms = sp.csr_matrix((m[2], (m[0], m[1])), shape=(n, n))
    assert sparse_rel_err(Mf, embed(op.assemble_matrix(w)) + Ms) < 1e-12
    assert nm == len(mesh.nodes)
