"""Extract a small MSH 2.2 binary fixture from a mesh the reference ships that Gmsh wrote in the
binary form, mesh/sr71_pure_hex.msh: its physical names, the first CELLS hexahedra (Gmsh type 5)
with their element ids and tags, the boundary quadrilaterals (type 3) whose nodes all belong to
those hexahedra, and those nodes with their Gmsh ids, in the file's own binary record layout
(little-endian int32 ids and tags, float64 coordinates).

    python tests/golden/make_gmsh_binary.py [/path/to/reference]
"""

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
CELLS = 600


def blocks(data):
    """(node records, element blocks [(type, ntags, records)], physical-name lines) of an MSH 2.2
    binary file."""
    pos = data.index(b"$PhysicalNames\n") + len(b"$PhysicalNames\n")
    end = data.index(b"$EndPhysicalNames", pos)
    names = data[pos:end].decode().strip().splitlines()
    pos = data.index(b"$Nodes\n") + len(b"$Nodes\n")
    nl = data.index(b"\n", pos)
    count = int(data[pos:nl])
    rec = np.dtype([("id", "<i4"), ("xyz", "<f8", (3,))])
    nodes = np.frombuffer(data, rec, count, nl + 1)
    pos = data.index(b"$Elements\n") + len(b"$Elements\n")
    nl = data.index(b"\n", pos)
    count, pos, seen, out = int(data[pos:nl]), nl + 1, 0, []
    per_type = {2: 3, 3: 4, 4: 4, 5: 8, 6: 6, 15: 1, 1: 2}
    while seen < count:
        etype, num, ntags = np.frombuffer(data, "<i4", 3, pos)
        pos += 12
        width = 1 + int(ntags) + per_type[int(etype)]
        recs = np.frombuffer(data, "<i4", int(num) * width, pos).reshape(int(num), width)
        pos += recs.nbytes
        out.append((int(etype), int(ntags), recs))
        seen += int(num)
    return nodes, out, names


def main(ref):
    data = (Path(ref) / "mesh" / "sr71_pure_hex.msh").read_bytes()
    nodes, elems, names = blocks(data)
    hexes = np.concatenate([r for t, _, r in elems if t == 5])[:CELLS]
    ntags = [n for t, n, _ in elems if t == 5][0]
    used = np.unique(hexes[:, 1 + ntags:])
    quads = np.concatenate([r for t, _, r in elems if t == 3])
    qt = [n for t, n, _ in elems if t == 3][0]
    quads = quads[np.all(np.isin(quads[:, 1 + qt:], used), axis=1)]
    keep = nodes[np.isin(nodes["id"], used)]
    out = [b"$MeshFormat\n2.2 1 8\n", np.array([1], "<i4").tobytes(), b"\n$EndMeshFormat\n",
           f"$PhysicalNames\n{len(names) - 1}\n".encode(), "\n".join(names[1:]).encode(), b"\n$EndPhysicalNames\n",
           f"$Nodes\n{len(keep)}\n".encode(), keep.tobytes(), b"\n$EndNodes\n",
           f"$Elements\n{len(hexes) + len(quads)}\n".encode()]
    for etype, nt, recs in ((5, ntags, hexes), (3, qt, quads)):
        if len(recs):
            out += [np.array([etype, len(recs), nt], "<i4").tobytes(), np.ascontiguousarray(recs).tobytes()]
    out.append(b"\n$EndElements\n")
    (HERE / "gmsh_sr71_binary.msh").write_bytes(b"".join(out))
    print(len(keep), "nodes,", len(hexes), "hexahedra,", len(quads), "boundary quadrilaterals")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
