"""Gmsh mesh I/O (pyfp3d/mesh/reader.py:19-300) without meshio.

``read_mesh`` parses MSH 2.2 files, ASCII or binary, into the reference's
structure-of-arrays ``Mesh``: nodes in file order (node tags renumbered
0..n-1 in order of appearance), tetrahedra in file order, boundary
triangles grouped by the name of their physical tag (an unnamed tag becomes
"surface_<tag>", untagged triangles "all_triangles"), and the tets'
physical tags with the volume names.  These are the conventions of the
reference's meshio-based reader (physical tag = an element's first tag,
cells of one type concatenated in file order).  ``write_mesh`` writes MSH
2.2 (binary by default) with one physical tag per boundary group, so a
round trip reproduces the groups.  Host code: mesh ingest happens once per
case.
"""

from __future__ import annotations

import struct
from pathlib import Path
from typing import Dict, List

import numpy as np

# nodes per element of the MSH 2.2 element types
_NODES_PER_TYPE = {1: 2, 2: 3, 3: 4, 4: 4, 5: 8, 6: 6, 7: 5, 8: 3, 9: 6, 10: 9, 11: 10, 12: 27,
                   13: 18, 14: 14, 15: 1, 16: 8, 17: 20, 18: 15, 19: 13}
_TRIANGLE, _TETRA = 2, 4


class Mesh:
    """Structure-of-arrays tetrahedral mesh (reader.py:19-83)."""

    def __init__(self):
        self.nodes = np.empty((0, 3), dtype=np.float64)
        self.elements = np.empty((0, 4), dtype=np.int32)
        self.boundary_faces: Dict[str, np.ndarray] = {}
        self.element_tags = np.empty(0, dtype=np.int32)
        self.tag_names: List[str] = []
        self.name = "unnamed"
        self.unit = "m"

    def __repr__(self) -> str:
        return (f"Mesh(n_nodes={len(self.nodes)}, n_tets={len(self.elements)}, "
                f"boundary_tags={list(self.boundary_faces.keys())})")

    def validate(self) -> bool:
        """Index and tag invariants (reader.py:52-83); AssertionError when
        one is violated."""
        n = len(self.nodes)
        assert np.all(np.isfinite(self.nodes)), "Non-finite node coordinates"
        assert np.all(self.elements >= 0), "Negative node index in element"
        assert np.all(self.elements < n), "Node index out of bounds"
        for tag, faces in self.boundary_faces.items():
            assert np.all(faces >= 0), f"Negative node in {tag} boundary"
            assert np.all(faces < n), f"Out-of-bounds node in {tag} boundary"
        if len(self.element_tags) > 0:
            assert len(self.element_tags) == len(self.elements), "Element tag count mismatch"
            assert np.all(self.element_tags >= 0), "Negative element tag"
            assert np.all(self.element_tags < len(self.tag_names)), "Tag out of range"
        return True


def _sections(data: bytes):
    """Yield (name, body bytes) of every $Section ... $EndSection."""
    pos = 0
    while True:
        start = data.find(b"$", pos)
        if start < 0:
            return
        eol = data.find(b"\n", start)
        name = data[start + 1:eol].strip().decode()
        end_tag = b"$End" + name.encode()
        end = data.find(end_tag, eol)
        if end < 0:
            raise ValueError(f"unterminated ${name} section")
        yield name, data[eol + 1:end]
        pos = end + len(end_tag)


def _parse_nodes(body: bytes, binary: bool, swap: bool):
    eol = body.find(b"\n")
    n = int(body[:eol])
    rest = body[eol + 1:]
    if binary:
        rec = np.dtype([("id", "<i4" if not swap else ">i4"), ("x", ("<f8" if not swap else ">f8"), 3)])
        arr = np.frombuffer(rest[:n * rec.itemsize], dtype=rec, count=n)
        return arr["id"].astype(np.int64), np.ascontiguousarray(arr["x"], dtype=np.float64)
    vals = np.array(rest.split(), dtype=np.float64).reshape(n, 4) if n else np.empty((0, 4))
    return vals[:, 0].astype(np.int64), np.ascontiguousarray(vals[:, 1:])


def _parse_elements(body: bytes, binary: bool, swap: bool):
    """[(type, physical tag, node tags)] per element, file order, as arrays
    grouped by type: {type: (phys (n,), nodes (n, k))}."""
    eol = body.find(b"\n")
    n = int(body[:eol])
    rest = body[eol + 1:]
    out: Dict[int, list] = {}
    if binary:
        it = ">i" if swap else "<i"
        pos, seen = 0, 0
        while seen < n:
            etype, count, ntags = struct.unpack_from(it[0] + "3i", rest, pos)
            pos += 12
            k = _NODES_PER_TYPE.get(etype)
            if k is None:
                raise ValueError(f"unsupported MSH element type {etype}")
            width = 1 + ntags + k
            blk = np.frombuffer(rest, dtype=it + "4", count=count * width, offset=pos).reshape(count, width)
            pos += 4 * count * width
            phys = blk[:, 1] if ntags > 0 else np.zeros(count, dtype=np.int32)
            out.setdefault(etype, []).append((phys.astype(np.int32), blk[:, 1 + ntags:].astype(np.int64)))
            seen += count
    else:
        for line in rest.splitlines()[:n]:
            v = [int(x) for x in line.split()]
            etype, ntags = v[1], v[2]
            k = _NODES_PER_TYPE.get(etype)
            if k is None:
                raise ValueError(f"unsupported MSH element type {etype}")
            phys = v[3] if ntags > 0 else 0
            out.setdefault(etype, []).append((np.array([phys], dtype=np.int32),
                                              np.array([v[3 + ntags:3 + ntags + k]], dtype=np.int64)))
    return {t: (np.concatenate([p for p, _ in b]), np.concatenate([c for _, c in b])) for t, b in out.items()}


def read_mesh(filepath, verbose: bool = False) -> Mesh:
    """Read a MSH 2.2 (ASCII or binary) tetrahedral mesh (reader.py:86-214).
    FileNotFoundError for a missing file; ValueError for another format
    version, an unsupported element type or a mesh without tetrahedra."""
    filepath = Path(filepath)
    if not filepath.exists():
        raise FileNotFoundError(f"Mesh file not found: {filepath}")
    data = filepath.read_bytes()
    binary = swap = False
    names: Dict[tuple, str] = {}
    node_ids = coords = elems = None
    for name, body in _sections(data):
        if name == "MeshFormat":
            head = body.split(b"\n", 1)
            version, ftype, dsize = head[0].split()
            if not version.startswith(b"2."):
                raise ValueError(f"MSH format {version.decode()} is not supported (MSH 2.2 only)")
            binary = int(ftype) == 1
            if binary:
                if int(dsize) != 8:
                    raise ValueError("binary MSH needs 8-byte reals")
                one = head[1][:4]
                swap = struct.unpack("<i", one)[0] != 1
        elif name == "PhysicalNames":
            lines = body.decode().splitlines()
            for line in lines[1:1 + int(lines[0])]:
                dim, tag, nm = line.split(maxsplit=2)
                names[(int(dim), int(tag))] = nm.strip().strip('"')
        elif name == "Nodes":
            node_ids, coords = _parse_nodes(body, binary, swap)
        elif name == "Elements":
            elems = _parse_elements(body, binary, swap)
    if coords is None or elems is None:
        raise ValueError("MSH file without $Nodes or $Elements")
    index = np.full(int(node_ids.max()) + 1 if len(node_ids) else 1, -1, dtype=np.int64)
    index[node_ids] = np.arange(len(node_ids))

    def remap(tags):
        if np.any(tags < 0) or np.any(tags >= len(index)) or np.any(index[tags] < 0):
            raise ValueError("element refers to an unknown node")
        return index[tags].astype(np.int32)

    if _TETRA not in elems or len(elems[_TETRA][1]) == 0:
        raise ValueError("Mesh must contain tetrahedral elements")
    mesh = Mesh()
    mesh.nodes = np.ascontiguousarray(coords, dtype=np.float64)
    tet_phys, tet_nodes = elems[_TETRA]
    mesh.elements = np.ascontiguousarray(remap(tet_nodes))
    if _TRIANGLE in elems:
        tri_phys, tri_nodes = elems[_TRIANGLE]
        tris = remap(tri_nodes)
        surf = {tag: nm for (dim, tag), nm in names.items() if dim == 2}
        if surf:
            for tag in np.unique(tri_phys):
                mesh.boundary_faces[surf.get(int(tag), f"surface_{int(tag)}")] = \
                    np.ascontiguousarray(tris[tri_phys == tag])
        else:
            mesh.boundary_faces["all_triangles"] = np.ascontiguousarray(tris)
    mesh.element_tags = tet_phys.astype(np.int32)
    vol = {tag: nm for (dim, tag), nm in names.items() if dim == 3}
    mesh.tag_names = ["bulk"]
    if vol:
        mesh.tag_names = [""] * (int(mesh.element_tags.max()) + 1)
        for tag, nm in vol.items():
            if tag < len(mesh.tag_names):
                mesh.tag_names[tag] = nm
    if len(mesh.element_tags) and int(mesh.element_tags.max()) >= len(mesh.tag_names):
        padded = [f"volume_{i}" for i in range(int(mesh.element_tags.max()) + 1)]
        padded[:len(mesh.tag_names)] = mesh.tag_names
        mesh.tag_names = padded
    mesh.name = filepath.stem
    mesh.validate()
    if verbose:
        print(f"Read mesh from {filepath}: {mesh}")
    return mesh


def write_mesh(mesh: Mesh, filepath, verbose: bool = False, binary: bool = True) -> None:
    """MSH 2.2 writer (reader.py:217-267): the tetrahedra with their
    element_tags as physical tags, then each boundary group as triangles
    with physical tag 1, 2, ... in group order, $PhysicalNames for every
    named volume tag and every group."""
    filepath = Path(filepath)
    tets = np.asarray(mesh.elements, dtype=np.int64)
    tet_tags = (np.asarray(mesh.element_tags, dtype=np.int64) if len(mesh.element_tags)
                else np.zeros(len(tets), dtype=np.int64))
    names = [(3, i, nm) for i, nm in enumerate(mesh.tag_names) if nm]
    blocks = [(_TETRA, tet_tags, tets)]
    for k, (nm, faces) in enumerate(mesh.boundary_faces.items(), start=1):
        names.append((2, k, nm))
        blocks.append((_TRIANGLE, np.full(len(faces), k, dtype=np.int64), np.asarray(faces, dtype=np.int64)))
    n_nodes = len(mesh.nodes)
    n_elem = sum(len(b[1]) for b in blocks)
    out = bytearray()
    out += b"$MeshFormat\n2.2 %d 8\n" % (1 if binary else 0)
    if binary:
        out += struct.pack("<i", 1) + b"\n"
    out += b"$EndMeshFormat\n"
    if names:
        out += b"$PhysicalNames\n%d\n" % len(names)
        for dim, tag, nm in names:
            out += f'{dim} {tag} "{nm}"\n'.encode()
        out += b"$EndPhysicalNames\n"
    out += b"$Nodes\n%d\n" % n_nodes
    ids = np.arange(1, n_nodes + 1)
    if binary:
        rec = np.zeros(n_nodes, dtype=[("id", "<i4"), ("x", "<f8", 3)])
        rec["id"], rec["x"] = ids, mesh.nodes
        out += rec.tobytes() + b"\n"
    else:
        out += "".join(f"{i} {x!r} {y!r} {z!r}\n" for i, (x, y, z) in zip(ids, mesh.nodes.tolist())).encode()
    out += b"$EndNodes\n$Elements\n%d\n" % n_elem
    eid = 1
    for etype, tags, conn in blocks:
        n, k = conn.shape
        if n == 0:
            continue
        rows = np.column_stack([np.arange(eid, eid + n), tags, np.zeros(n, dtype=np.int64), conn + 1])
        if binary:
            out += struct.pack("<3i", etype, n, 2) + rows.astype("<i4").tobytes()
        else:
            out += "".join(f"{r[0]} {etype} 2 {' '.join(str(v) for v in r[1:])}\n" for r in rows.tolist()).encode()
        eid += n
    if binary:
        out += b"\n"
    out += b"$EndElements\n"
    filepath.write_bytes(bytes(out))
    if verbose:
        print(f"Wrote mesh to {filepath}")


def mesh_stats(mesh: Mesh) -> Dict:
    """Node and element counts, tet volumes and the 6 E edge lengths
    (reader.py:270-300; volumes |det J| / 6 as mesh/metrics.py:27-92)."""
    X = mesh.nodes[mesh.elements.astype(np.int64)]
    J = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)
    vol = np.abs(np.linalg.det(J)) / 6.0
    pairs = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))
    edges = np.concatenate([np.linalg.norm(X[:, b] - X[:, a], axis=1)[:, None] for a, b in pairs], axis=1).ravel()
    return {"n_nodes": len(mesh.nodes), "n_elements": len(mesh.elements), "total_volume": float(vol.sum()),
            "min_volume": float(vol.min()), "max_volume": float(vol.max()), "mean_volume": float(vol.mean()),
            "min_edge_length": float(edges.min()), "max_edge_length": float(edges.max()),
            "mean_edge_length": float(edges.mean())}
