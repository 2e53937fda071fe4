"""``meshio`` stand-in: Gmsh 2.2 ASCII reader/writer for linear cells.

Returns the fields the reference's ``hybrid/mesh.py:186-205,343-359`` reads:
``points``, ``cells`` (blocks with ``type``/``data``), ``field_data`` and
``cell_data["gmsh:physical"]``.  Consecutive elements of one type form one
block, as meshio does.  First-order cell types need no node reordering between Gmsh
and meshio; second-order cells are passed through in the order they were written.
"""

from dataclasses import dataclass

import numpy as np

_GMSH_TYPES = {1: ("line", 2), 2: ("triangle", 3), 3: ("quad", 4), 4: ("tetra", 4),
               5: ("hexahedron", 8), 6: ("wedge", 6), 15: ("vertex", 1),
               # complete second-order cells, kept in the node order they were written in (the
               # fixture generators write meshio's order, so nothing is reordered here)
               11: ("tetra10", 10), 12: ("hexahedron27", 27), 13: ("wedge18", 18)}
_TYPE_IDS = {name: (tid, n) for tid, (name, n) in _GMSH_TYPES.items()}


@dataclass
class CellBlock:
    type: str
    data: np.ndarray


class Mesh:
    def __init__(self, points, cells, cell_data=None, field_data=None):
        self.points = np.asarray(points, dtype=np.float64)
        self.cells = [c if isinstance(c, CellBlock) else CellBlock(c[0], np.asarray(c[1]))
                      for c in cells]
        self.cell_data = cell_data or {}
        self.field_data = field_data or {}


def read(path):
    with open(path) as handle:
        lines = [line.strip() for line in handle]
    field_data, points, blocks, physical = {}, None, [], []
    i = 0
    while i < len(lines):
        line = lines[i]
        if line == "$PhysicalNames":
            count = int(lines[i + 1])
            for k in range(count):
                dim, tag, name = lines[i + 2 + k].split(maxsplit=2)
                field_data[name.strip('"')] = np.array([int(tag), int(dim)])
            i += count + 2
        elif line == "$Nodes":
            count = int(lines[i + 1])
            rows = np.array([lines[i + 2 + k].split() for k in range(count)], dtype=np.float64)
            ids = rows[:, 0].astype(np.int64)
            points = np.zeros((int(ids.max()), 3))
            points[ids - 1] = rows[:, 1:4]
            i += count + 2
        elif line == "$Elements":
            count = int(lines[i + 1])
            current_type, current, current_tags = None, [], []
            for k in range(count):
                parts = [int(v) for v in lines[i + 2 + k].split()]
                etype, ntags = parts[1], parts[2]
                tags = parts[3:3 + ntags]
                nodes = parts[3 + ntags:]
                name = _GMSH_TYPES[etype][0]
                if name != current_type and current:
                    blocks.append(CellBlock(current_type, np.asarray(current, dtype=np.int64) - 1))
                    physical.append(np.asarray(current_tags, dtype=np.int64))
                    current, current_tags = [], []
                current_type = name
                current.append(nodes)
                current_tags.append(tags[0] if tags else 0)
            if current:
                blocks.append(CellBlock(current_type, np.asarray(current, dtype=np.int64) - 1))
                physical.append(np.asarray(current_tags, dtype=np.int64))
            i += count + 2
        else:
            i += 1
    return Mesh(points, blocks, {"gmsh:physical": physical}, field_data)


def write_gmsh22(path, points, cells, physical, field_data):
    """cells: list of (type, array); physical: list of per-cell tag arrays."""
    out = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", str(len(field_data))]
    for name, (tag, dim) in field_data.items():
        out.append(f'{dim} {tag} "{name}"')
    out += ["$EndPhysicalNames", "$Nodes", str(len(points))]
    for k, p in enumerate(points):
        out.append(f"{k + 1} {float(p[0])!r} {float(p[1])!r} {float(p[2])!r}")
    out += ["$EndNodes", "$Elements", str(sum(len(c[1]) for c in cells))]
    eid = 1
    for (name, data), tags in zip(cells, physical):
        tid = _TYPE_IDS[name][0]
        for row, tag in zip(np.asarray(data), np.asarray(tags)):
            out.append(f"{eid} {tid} 2 {int(tag)} {int(tag)} " + " ".join(str(int(v) + 1) for v in row))
            eid += 1
    out += ["$EndElements"]
    with open(path, "w") as handle:
        handle.write("\n".join(out) + "\n")
