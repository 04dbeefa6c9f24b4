"""Gmsh ingest (pyfp3d/mesh/reader.py:19-300) and the real-geometry
lifting case: the NACA0012 2.5D coarse mesh as read by
up3d_b200.mesh.reader (tests/golden/naca_coarse.npz, pinned at generation
time against the reference's committed mesh statistics), MSH 2.2 round
trips, reader errors, and the oracle's exact-step coupled Newton against
the reference's solve_newton_lifting on the reference's own wake cut."""

import numpy as np
import pytest

from conftest import GOLDEN


@pytest.fixture(scope="module")
def naca():
    return np.load(GOLDEN / "naca_coarse.npz")


def _mesh(g):
    from up3d_b200.mesh.reader import Mesh
    m = Mesh()
    m.nodes, m.elements = g["nodes"], g["elements"]
    m.boundary_faces = {k.split("/", 1)[1]: g[k].astype(np.int32) for k in g.files if k.startswith("faces/")}
    m.element_tags = np.zeros(len(m.elements), dtype=np.int32)
    m.tag_names = ["fluid"]
    return m


def test_mesh_stats_match_reference(naca):
    from up3d_b200.mesh.reader import mesh_stats
    ref = dict(zip(naca["stats_keys"].tolist(), naca["stats_values"].tolist()))
    st = mesh_stats(_mesh(naca))
    for k, v in st.items():
        assert abs(v - ref[k]) <= 1e-12 * abs(ref[k]), k
    assert len(naca["faces/wake"]) == ref["n_wake_faces"]


@pytest.mark.parametrize("binary", [True, False])
def test_msh22_round_trip(naca, tmp_path, binary):
    from up3d_b200.mesh.reader import read_mesh, write_mesh
    m = _mesh(naca)
    path = tmp_path / ("m_bin.msh" if binary else "m_asc.msh")
    write_mesh(m, path, binary=binary)
    r = read_mesh(path)
    assert np.array_equal(r.nodes, m.nodes)
    assert np.array_equal(r.elements, m.elements)
    assert list(r.boundary_faces) == list(m.boundary_faces)
    for k in m.boundary_faces:
        assert np.array_equal(r.boundary_faces[k], m.boundary_faces[k])
    assert r.tag_names == ["fluid"] and np.all(r.element_tags == 0)
    assert r.name == path.stem


def test_reader_rejects_bad_input(tmp_path):
    from up3d_b200.mesh.reader import read_mesh
    with pytest.raises(FileNotFoundError):
        read_mesh(tmp_path / "missing.msh")
    p = tmp_path / "v4.msh"
    p.write_text("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n")
    with pytest.raises(ValueError):
        read_mesh(p)
    p = tmp_path / "tri.msh"
    p.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n3\n1 0 0 0\n2 1 0 0\n3 0 1 0\n$EndNodes\n"
                 "$Elements\n1\n1 2 2 0 0 1 2 3\n$EndElements\n")
    with pytest.raises(ValueError):
        read_mesh(p)


def test_reader_ascii_node_tags_renumbered(tmp_path):
    """Non-contiguous node tags map to 0..n-1 in order of appearance; an
    unnamed surface tag becomes surface_<tag>."""
    from up3d_b200.mesh.reader import read_mesh
    p = tmp_path / "tags.msh"
    p.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$PhysicalNames\n1\n3 7 \"air\"\n$EndPhysicalNames\n"
                 "$Nodes\n4\n10 0 0 0\n20 1 0 0\n30 0 1 0\n40 0 0 1\n$EndNodes\n"
                 "$Elements\n2\n1 4 2 7 1 10 20 30 40\n2 2 2 5 1 40 20 10\n$EndElements\n")
    m = read_mesh(p)
    assert np.array_equal(m.elements, [[0, 1, 2, 3]])
    assert list(m.boundary_faces) == ["all_triangles"]
    assert np.array_equal(m.boundary_faces["all_triangles"], [[3, 1, 0]])
    assert m.tag_names[7] == "air" and m.element_tags.tolist() == [7]


def naca_cut(g):
    from up3d_b200.mesh.wake_cut import load_cut
    return load_cut(g)


@pytest.mark.parametrize("case", ["m05", "m07"])
def test_oracle_naca_lifting_solve_matches_reference(naca, case):
    from oracle import oracle as O
    from up3d_b200.constraints.dirichlet import FarfieldBasis, freestream_phi
    mc, wc = naca_cut(naca)
    m_inf, alpha = float(naca[case + "/m_inf"]), float(naca[case + "/alpha_deg"])
    basis = FarfieldBasis(mc, wc, alpha, 1.0)
    vals0, V = basis.at_mach(float(np.sqrt(1.0 - m_inf ** 2)))
    sysm = O.LiftingSystem(mc.nodes, mc.elements, wc, basis.dir_red, vals0, V)
    phi0 = freestream_phi(mc.nodes[:sysm.n_red], alpha, 1.0)
    phi, gamma, hist, ok = sysm.solve(phi0[sysm.free], np.zeros(sysm.n_st), m_inf)
    assert ok and len(hist) - 1 == int(naca[case + "/n_newton"])
    assert np.max(np.abs(phi - naca[case + "/phi"])) <= 1e-10
    assert np.max(np.abs(gamma - naca[case + "/gamma"])) <= 1e-10
    f = O.wall_force_coefficients(mc.nodes, mc.elements, np.asarray(mc.boundary_faces["wall"]), phi,
                                  alpha_deg=alpha, m_inf=m_inf)
    assert np.max(np.abs(f["cp_tri"] - naca[case + "/cp_tri"])) <= 1e-8
    assert abs(f["cl"] - float(naca[case + "/cl"])) <= 1e-10


def test_naca_medium_mesh_stats_match_reference():
    from up3d_b200.mesh.reader import Mesh, mesh_stats
    g = np.load(GOLDEN / "naca_medium_mesh.npz")
    m = Mesh()
    m.nodes, m.elements = g["nodes"], g["elements"]
    ref = dict(zip(g["stats_keys"].tolist(), g["stats_values"].tolist()))
    for k, v in mesh_stats(m).items():
        assert abs(v - ref[k]) <= 1e-12 * abs(ref[k]), k


def test_cut_wake_matches_reference_on_naca(naca):
    """cut_wake on the NACA mesh reproduces the reference's own cut
    (mesh/wake_cut.py:225-441) array for array."""
    from up3d_b200.mesh.wake_cut import cut_arrays, cut_wake
    mc, wc = cut_wake(_mesh(naca))
    got = cut_arrays(mc, wc)
    ref_keys = [k for k in naca.files if k.startswith(("cut/", "wc/"))]
    assert sorted(got) == sorted(ref_keys)
    for k in ref_keys:
        assert np.array_equal(np.asarray(got[k]), naca[k]), k


def test_cut_wake_rejects_bad_sheets(naca):
    from up3d_b200.mesh.wake_cut import cut_wake
    m = _mesh(naca)
    with pytest.raises(ValueError):
        cut_wake(m, wake_tag="nope")
    bad = _mesh(naca)
    bad.boundary_faces["wake"] = bad.boundary_faces["wall"][:4]     # boundary faces: one owner each
    with pytest.raises(AssertionError):
        cut_wake(bad)
    with pytest.raises(AssertionError):
        cut_wake(m, upper_hint=(0.0, 0.0, 1.0))                     # sides not separable along z


def test_cut_wake_matches_reference_on_swept_part_span_sheet():
    """A swept, part-span sheet (several stations, interior free-edge nodes
    kept single-valued): cut_wake reproduces the reference's cut
    (tests/golden/swept_cut.npz)."""
    from up3d_b200.mesh.reader import Mesh
    from up3d_b200.mesh.wake_cut import cut_arrays, cut_wake
    g = np.load(GOLDEN / "swept_cut.npz")
    m = Mesh()
    m.nodes, m.elements = g["nodes"], g["elements"]
    m.boundary_faces = {k.split("/", 1)[1]: g[k].astype(np.int32) for k in g.files if k.startswith("faces/")}
    m.element_tags = np.zeros(len(m.elements), dtype=np.int32)
    m.tag_names = ["fluid"]
    m.name = "swept_sheet"
    mc, wc = cut_wake(m)
    assert wc.n_stations == 3 and len(wc.free_nodes) == 13
    got = cut_arrays(mc, wc)
    ref_keys = [k for k in g.files if k.startswith(("cut/", "wc/"))]
    assert sorted(got) == sorted(ref_keys)
    for k in ref_keys:
        assert np.array_equal(np.asarray(got[k]), g[k]), k


def test_cut_wake_on_naca_medium():
    """cut_wake on the NACA medium mesh (61,788 tets, 984 wake faces): the
    topology asserts hold and every sheet node is duplicated."""
    from up3d_b200.mesh.reader import Mesh
    from up3d_b200.mesh.wake_cut import cut_wake
    g = np.load(GOLDEN / "naca_medium_mesh.npz")
    m = Mesh()
    m.nodes, m.elements = g["nodes"], g["elements"]
    m.boundary_faces = {k.split("/", 1)[1]: g[k] for k in g.files if k.startswith("faces/")}
    m.element_tags = np.zeros(len(m.elements), dtype=np.int32)
    m.tag_names = ["fluid"]
    mc, wc = cut_wake(m)
    assert len(wc.slave_nodes) == len(np.unique(m.boundary_faces["wake"])) and wc.n_stations == 1
    assert len(mc.nodes) == len(m.nodes) + len(wc.slave_nodes)


@pytest.mark.parametrize("beta", [1.0, 0.8])
def test_spanwise_farfield_matches_reference(beta):
    """farfield_dirichlet with the spanwise vortex strength on the swept
    part-span cut (Gamma(z) interpolated over three stations, anchored to 0
    at the sheet tip inside the span; constraints/dirichlet.py:98-182)."""
    from up3d_b200.constraints.dirichlet import farfield_dirichlet
    from up3d_b200.mesh.wake_cut import load_cut
    g = np.load(GOLDEN / "swept_cut.npz")
    mc, wc = load_cut(g)
    dn, dv = farfield_dirichlet(mc, wc, 2.0, g["ff_gamma"], 1.0, tuple(g["ff_vortex_center"]), beta=beta,
                                spanwise_gamma=True)
    assert np.array_equal(dn, g[f"ff_beta{beta}/nodes"])
    assert np.array_equal(dv, g[f"ff_beta{beta}/values"])
