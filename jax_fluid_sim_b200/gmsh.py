"""Gmsh mesh files (MSH 2.2 ASCII or binary, MSH 4.1 ASCII) into a ``MeshSource``.

The reference reads its meshes with meshio (hybrid/mesh.py:182-236, mesh_loader.py).  This
reader keeps what the hybrid path uses: node coordinates, the physical names and, per cell
block, the cells and their physical tags.  Element types follow the reference's aliases
(hybrid/mesh.py:11-20): tetrahedra, wedges and hexahedra of first order, and the serendipity
hexahedron20 / wedge15, whose corner nodes come first; boundary triangles and quadrilaterals
(and their second-order forms) keep their corners.  The complete second-order cells tetra10,
wedge18 and hexahedron27 carry curved geometry: their nodes are reordered from Gmsh's numbering
to meshio's (the order ``HybridMesh`` and the reference's P2 permutations take).  The
reordering is not a stored table: each node is placed at its reference coordinates under both
numberings (Gmsh's from its documented edge, face and centre nodes; meshio's from the
second-order reference element's nodes and the P2 permutations) and matched by position.
"""
from pathlib import Path

import numpy as np

from . import _native
from .meshgen import MeshSource

# Gmsh element type -> (cell type name, corner count, total node count)
_TYPES = {
    2: ("triangle", 3, 3), 3: ("quad", 4, 4), 4: ("tetra", 4, 4), 5: ("hexahedron", 8, 8), 6: ("wedge", 6, 6),
    9: ("triangle", 3, 6), 10: ("quad", 4, 9), 16: ("quad", 4, 8), 17: ("hexahedron", 8, 20),
    18: ("wedge", 6, 15), 1: (None, 2, 2), 8: (None, 2, 3), 15: (None, 1, 1),
}
_CURVED = {11: "tetra10", 12: "hexahedron27", 13: "wedge18"}
# Gmsh's complete second-order cells: the corner nodes of the first-order cell, then one node at
# the midpoint of each listed edge, at the centre of each listed quadrilateral face and, for the
# hexahedron, at the cell centre (Gmsh reference manual, node ordering of the reference elements).
_GMSH_P2 = {
    "tetra10": ("tetra", ((0, 1), (1, 2), (2, 0), (3, 0), (3, 2), (3, 1)), (), False),
    "wedge18": ("wedge", ((0, 1), (0, 2), (0, 3), (1, 2), (1, 4), (2, 5), (3, 4), (3, 5), (4, 5)),
                ((0, 1, 4, 3), (0, 2, 5, 3), (1, 2, 5, 4)), False),
    "hexahedron27": ("hexahedron", ((0, 1), (0, 3), (0, 4), (1, 2), (1, 5), (2, 3), (2, 6), (3, 7), (4, 5),
                                    (4, 7), (5, 6), (6, 7)),
                     ((0, 1, 2, 3), (0, 1, 5, 4), (0, 3, 7, 4), (1, 2, 6, 5), (2, 3, 7, 6), (4, 5, 6, 7)), True),
}


def _gmsh_p2_points(ctype):
    from .reference import CORNERS
    etype, edges, faces, centre = _GMSH_P2[ctype]
    c = CORNERS[etype]
    pts = list(c) + [0.5 * (c[a] + c[b]) for a, b in edges] + [c[list(f)].mean(axis=0) for f in faces]
    if centre:
        pts.append(c.mean(axis=0))
    return np.asarray(pts)


def _meshio_p2_points(ctype):
    from .mesh import P2_PERMUTATIONS
    from .reference import RefElement
    etype = _GMSH_P2[ctype][0]
    nodes = RefElement(etype, 2).nodes                 # reference node r is meshio node perm[r]
    out = np.empty_like(nodes)
    out[P2_PERMUTATIONS[ctype]] = nodes
    return out


def gmsh_to_meshio(ctype):
    """Column order taking a complete second-order cell's Gmsh node list to meshio's:
    meshio_cells = gmsh_cells[:, gmsh_to_meshio(ctype)]."""
    g, m = _gmsh_p2_points(ctype), _meshio_p2_points(ctype)
    d = np.linalg.norm(m[:, None, :] - g[None, :, :], axis=-1)
    order = np.argmin(d, axis=1)
    if len(g) != len(m) or not np.array_equal(np.sort(order), np.arange(len(g))) or d.min(axis=1).max() > 1e-12:
        raise AssertionError(f"{ctype}: Gmsh and meshio node positions do not match one to one")
    return order.astype(np.int64)
_ORDER = ("hexahedron", "hexahedron27", "wedge", "wedge18", "tetra", "tetra10", "quad", "triangle")


def _ascii_sections(data):
    """{name: body bytes} of an ASCII mesh: the bytes between a "$Name" line and its "$EndName"."""
    out, pos, n = {}, 0, len(data)
    while pos < n:
        eol = data.find(b"\n", pos)
        eol = n if eol < 0 else eol
        line = data[pos:eol].strip()
        if line.startswith(b"$") and not line.startswith(b"$End"):
            tag = b"\n$End" + line[1:]
            end = data.find(tag, eol)
            if end < 0:
                raise ValueError(f"section {line.decode('ascii', 'replace')} has no end")
            out[line[1:].decode("ascii", "replace")] = data[eol + 1:end + 1]
            eol = data.find(b"\n", end + 1)
            eol = n if eol < 0 else eol
        pos = eol + 1
    return out


def _lines(body):
    return body.decode("ascii", "replace").splitlines() if body is not None else None


def _physical_names(sec):
    names = {}
    for line in sec[1:1 + int(sec[0])] if sec else []:
        parts = line.split(maxsplit=2)
        names[parts[2].strip().strip('"')] = (int(parts[1]), int(parts[0]))
    return names


def _assemble(points, node_index, records):
    """records: list of (gmsh type, physical tag, node tags array (n, k))."""
    grouped = {}
    for etype, phys, nodes in records:
        if etype in _CURVED:
            name = _CURVED[etype]
            conn = node_index[nodes[:, gmsh_to_meshio(name)]]
        elif etype in _TYPES:
            name, corners, _ = _TYPES[etype]
            if name is None:
                continue
            conn = node_index[nodes[:, :corners]]
        else:
            raise ValueError(f"unsupported Gmsh element type {etype}")
        grouped.setdefault(name, ([], []))
        grouped[name][0].append(conn)
        grouped[name][1].append(np.broadcast_to(np.asarray(phys, np.int32), (len(conn),)))
    if not any(t in grouped for t in ("hexahedron", "wedge", "tetra", "hexahedron27", "wedge18", "tetra10")):
        raise ValueError("Mesh contains no tetrahedron, wedge, or hexahedron")
    cells = [(t, np.concatenate(grouped[t][0]).astype(np.int32)) for t in _ORDER if t in grouped]
    phys = [np.concatenate(grouped[t][1]).astype(np.int32) for t in _ORDER if t in grouped]
    return cells, phys


def _records(etype, phys, offsets, nodes):
    """(gmsh type, physical tag, node ids (n, k)) per (type, tag) pair in the order the pairs first
    appear, each pair's elements in file order."""
    key = (etype.astype(np.int64) << 32) | (phys.astype(np.int64) & 0xFFFFFFFF)
    _, first, inv = np.unique(key, return_index=True, return_inverse=True)
    out = []
    for g in np.argsort(first, kind="stable"):
        rows = np.flatnonzero(inv == g)
        k = offsets[rows + 1] - offsets[rows]
        if np.any(k != k[0]):
            raise ValueError(f"Gmsh element type {int(etype[rows[0]])} has records of different lengths")
        out.append((int(etype[rows[0]]), int(phys[rows[0]]), nodes[offsets[rows][:, None] + np.arange(k[0])]))
    return out


def _node_index(ids):
    index = np.full(ids.max() + 1, -1, np.int64)
    index[ids] = np.arange(len(ids))
    return index


def _read_v2(sec):
    """MSH 2.2 ASCII: the node and element records parsed on the host (``dgb_msh2_*``)."""
    head, _, body = sec["Nodes"].partition(b"\n")
    ids, xyz = _native.msh_nodes(body, int(head), 2)
    head, _, body = sec["Elements"].partition(b"\n")
    etype, phys, offsets, nodes = _native.msh_elements(body, int(head), 2, len(body) // 2 + 1)
    return xyz, _node_index(ids), _records(etype, phys, offsets, nodes)


def _read_v4(sec):
    """MSH 4.1 ASCII: the entities' physical tags here, the node and element blocks parsed on the
    host (``dgb_msh4_*``)."""
    phys_of = {}
    ent = _lines(sec.get("Entities"))
    if ent:
        counts = [int(x) for x in ent[0].split()]
        row = 1
        for dim, count in enumerate(counts):
            for _ in range(count):
                v = ent[row].split()
                row += 1
                tag = int(v[0])
                nfix = 4 if dim == 0 else 7              # point: tag x y z; others: tag + bounding box
                nphys = int(v[nfix])
                phys_of[(dim, tag)] = int(v[nfix + 1]) if nphys > 0 else 0
    body = sec["Nodes"]
    ids, xyz = _native.msh_nodes(body, int(body.split(None, 2)[1]), 4)
    body = sec["Elements"]
    etype, edim, etag, offsets, nodes = _native.msh_elements(body, int(body.split(None, 2)[1]), 4,
                                                             len(body) // 2 + 1)
    ent_key = (edim.astype(np.int64) << 32) | (etag.astype(np.int64) & 0xFFFFFFFF)
    uniq, inv = np.unique(ent_key, return_inverse=True)
    phys = np.asarray([phys_of.get((int(u >> 32), int(np.int32(u & 0xFFFFFFFF))), 0) for u in uniq],
                      np.int32)[inv] if len(uniq) else np.zeros(0, np.int32)
    return xyz, _node_index(ids), _records(etype, phys, offsets, nodes)


def _node_count(etype):
    if etype in _CURVED:
        return {"tetra10": 10, "hexahedron27": 27, "wedge18": 18}[_CURVED[etype]]
    if etype in _TYPES:
        return _TYPES[etype][2]
    raise ValueError(f"unsupported Gmsh element type {etype}")


def _read_v2_binary(data):
    """MSH 2.2 binary (Gmsh reference manual, legacy MSH 2 format): the section headers, the
    physical names and the counts are text lines; after the format line one int 1 gives the byte
    order; the nodes are records (int id, 3 doubles); the elements come in blocks, each a header
    (int type, int count, int number of tags) followed by count records (int id, the tags, the
    node ids)."""
    pos = 0

    def line():
        nonlocal pos
        end = data.index(b"\n", pos)
        out = data[pos:end].decode("ascii", "replace").strip()
        pos = end + 1
        return out

    def skip_to(tag):
        nonlocal pos
        pos = data.index(tag, pos) + len(tag)
        if pos < len(data) and data[pos:pos + 1] == b"\r":
            pos += 1
        if pos < len(data) and data[pos:pos + 1] == b"\n":
            pos += 1

    order, field, nodes, records = "<", {}, None, []
    while pos < len(data):
        head = line()
        if not head.startswith("$"):
            continue
        name = head[1:]
        if name == "MeshFormat":
            version, binary, dsize = line().split()[:3]
            if int(dsize) != 8:
                raise NotImplementedError("binary MSH files need 8-byte reals")
            one = data[pos:pos + 4]
            order = "<" if np.frombuffer(one, "<i4")[0] == 1 else ">"
            pos += 4
            skip_to(b"$EndMeshFormat")
        elif name == "PhysicalNames":
            count = int(line())
            field = _physical_names([str(count)] + [line() for _ in range(count)])
            skip_to(b"$EndPhysicalNames")
        elif name == "Nodes":
            count = int(line())
            rec = np.dtype([("id", order + "i4"), ("xyz", order + "f8", (3,))])
            nodes = np.frombuffer(data, rec, count, pos)
            pos += count * rec.itemsize
            skip_to(b"$EndNodes")
        elif name == "Elements":
            count = int(line())
            seen, by_shape = 0, {}
            while seen < count:
                etype, num, ntags = (int(v) for v in np.frombuffer(data, order + "i4", 3, pos))
                pos += 12
                k = _node_count(etype)
                block = np.frombuffer(data, order + "i4", num * (1 + ntags + k), pos).reshape(num, 1 + ntags + k)
                pos += block.nbytes
                phys = block[:, 1] if ntags > 0 else np.zeros(num, np.int32)
                for p in np.unique(phys).tolist():
                    by_shape.setdefault((etype, p), []).append(block[phys == p, 1 + ntags:])
                seen += num
            records = [(t, p, np.concatenate(n).astype(np.int64)) for (t, p), n in by_shape.items()]
            skip_to(b"$EndElements")
        else:
            skip_to(b"$End" + name.encode())
    if nodes is None:
        raise ValueError("the mesh has no $Nodes section")
    ids = nodes["id"].astype(np.int64)
    index = np.full(ids.max() + 1, -1, np.int64)
    index[ids] = np.arange(len(ids))
    return np.ascontiguousarray(nodes["xyz"], np.float64), index, records, field


def read_msh(path, periodic_map=None):
    """Read a Gmsh MSH 2.2 (ASCII or binary) or 4.1 ASCII file into a ``MeshSource`` (optionally
    with a periodic point map for ``HybridMesh``)."""
    data = Path(path).read_bytes()
    if not data.lstrip().startswith(b"$MeshFormat"):
        raise ValueError(f"{path} is not a Gmsh mesh")
    fmt = data.split(b"\n", 2)[1].split()
    if len(fmt) >= 2 and int(fmt[1]) != 0:
        if not fmt[0].decode().startswith("2"):
            raise NotImplementedError("binary MSH files are read in version 2.2 only; save 4.1 files as ASCII")
        points, index, records, field = _read_v2_binary(data)
        cells, phys = _assemble(points, index, records)
        return MeshSource(points, cells, phys, field, periodic_map)
    sec = _ascii_sections(data)
    if "MeshFormat" not in sec:
        raise ValueError(f"{path} is not a Gmsh mesh")
    version, binary = _lines(sec["MeshFormat"])[0].split()[:2]
    field = _physical_names(_lines(sec.get("PhysicalNames")))
    if version.startswith("2"):
        points, index, records = _read_v2(sec)
    elif version.startswith("4"):
        points, index, records = _read_v4(sec)
    else:
        raise NotImplementedError(f"MSH version {version}")
    cells, phys = _assemble(points, index, records)
    return MeshSource(points, cells, phys, field, periodic_map)


def write_msh22(path, source, binary=False):
    """Write a ``MeshSource`` as an MSH 2.2 file, ASCII or binary (first-order cells, and complete
    second-order cells given in meshio's node order, written in Gmsh's)."""
    codes = {"triangle": 2, "quad": 3, "tetra": 4, "hexahedron": 5, "wedge": 6,
             "tetra10": 11, "hexahedron27": 12, "wedge18": 13}
    if binary:
        return _write_msh22_binary(path, source, codes)
    out = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", str(len(source.field_data))]
    for name, (tag, dim) in source.field_data.items():
        out.append(f'{dim} {tag} "{name}"')
    out += ["$EndPhysicalNames", "$Nodes", str(len(source.points))]
    out += [f"{i + 1} {x!r} {y!r} {z!r}" for i, (x, y, z) in enumerate(np.asarray(source.points, float).tolist())]
    out += ["$EndNodes", "$Elements", str(sum(len(c) for _, c in source.cells))]
    k = 1
    for (ctype, conn), phys in zip(source.cells, source.physical):
        conn = np.asarray(conn)
        if ctype in _GMSH_P2:
            to_gmsh = np.empty(conn.shape[1], np.int64)
            to_gmsh[gmsh_to_meshio(ctype)] = np.arange(conn.shape[1])
            conn = conn[:, to_gmsh]
        for cell, p in zip(conn, np.asarray(phys)):
            out.append(f"{k} {codes[ctype]} 2 {int(p)} {int(p)} " + " ".join(str(int(v) + 1) for v in cell))
            k += 1
    out.append("$EndElements")
    Path(path).write_text("\n".join(out) + "\n")


def _write_msh22_binary(path, source, codes):
    out = [b"$MeshFormat\n2.2 1 8\n", np.array([1], "<i4").tobytes(), b"\n$EndMeshFormat\n",
           f"$PhysicalNames\n{len(source.field_data)}\n".encode()]
    for name, (tag, dim) in source.field_data.items():
        out.append(f'{dim} {tag} "{name}"\n'.encode())
    pts = np.asarray(source.points, np.float64)
    rec = np.zeros(len(pts), np.dtype([("id", "<i4"), ("xyz", "<f8", (3,))]))
    rec["id"] = np.arange(1, len(pts) + 1)
    rec["xyz"] = pts
    out += [b"$EndPhysicalNames\n", f"$Nodes\n{len(pts)}\n".encode(), rec.tobytes(), b"\n$EndNodes\n",
            f"$Elements\n{sum(len(c) for _, c in source.cells)}\n".encode()]
    k = 1
    for (ctype, conn), phys in zip(source.cells, source.physical):
        conn = np.asarray(conn, np.int64)
        if ctype in _GMSH_P2:
            to_gmsh = np.empty(conn.shape[1], np.int64)
            to_gmsh[gmsh_to_meshio(ctype)] = np.arange(conn.shape[1])
            conn = conn[:, to_gmsh]
        n = len(conn)
        if n == 0:
            continue
        block = np.empty((n, 3 + conn.shape[1]), "<i4")
        block[:, 0] = np.arange(k, k + n)
        block[:, 1] = block[:, 2] = np.asarray(phys, np.int64)
        block[:, 3:] = conn + 1
        out += [np.array([codes[ctype], n, 2], "<i4").tobytes(), block.tobytes()]
        k += n
    out.append(b"\n$EndElements\n")
    Path(path).write_bytes(b"".join(out))


read_gmsh = read_msh     # the name HybridMesh(path) uses
