"""Type-blocked mesh topology: element blocks and face pairing.

Oracle restatement of ``hybrid/mesh.py``:
* element blocks in hex -> wedge -> tet order; corners for the topology, and for the complete
  second-order cells (tetra10, wedge18, hexahedron27) their geometry nodes permuted from
  meshio order to the reference element's node order (``hybrid/mesh.py:11-35,240-286``);
* cell centres/volumes from a fixed tetrahedral decomposition (``:61-76,207-238``);
* face pairing by sorted corner ids in visiting order, owner = first visitor,
  unpaired faces tagged from boundary cells (``:343-359,378-405``);
* face centre/normal/area from the owner's corners, normal flipped toward the
  neighbour centre (``:361-376,417-443``);
* validation (``:461-477``).

Extension (not in the reference): ``periodic_map`` sends every point id to a
canonical id; face keys use canonical ids, so faces on opposite periodic
planes pair.  For a periodic pair the neighbour-centre flip is skipped (the
centre displacement wraps around the domain); the owner-outward normal stands.
"""

from dataclasses import dataclass, field

import numpy as np

ALIASES = {"tetra": ("tetra", 4), "tetra10": ("tetra", 4), "wedge": ("wedge", 6), "wedge15": ("wedge", 6),
           "wedge18": ("wedge", 6), "hexahedron": ("hexahedron", 8), "hexahedron20": ("hexahedron", 8),
           "hexahedron27": ("hexahedron", 8)}
P2_PERMUTATIONS = {
    "tetra10": [0, 1, 2, 3, 4, 6, 7, 5, 8, 9],
    "wedge18": [0, 1, 2, 6, 9, 7, 3, 4, 5, 12, 14, 13, 8, 10, 11, 15, 17, 16],
    "hexahedron27": [0, 1, 8, 3, 2, 10, 11, 9, 24, 4, 5, 12, 7, 6, 14, 15, 13, 25, 16, 17, 22, 19, 18, 23, 20, 21,
                     26],
}
LOCAL_FACES = {
    "tetra": ((0, 2, 1), (0, 1, 3), (1, 2, 3), (2, 0, 3)),
    "wedge": ((0, 2, 1), (3, 4, 5), (0, 1, 4, 3), (1, 2, 5, 4), (2, 0, 3, 5)),
    "hexahedron": ((0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)),
}
TETRA_DECOMPOSITIONS = {
    "tetra": ((0, 1, 2, 3),),
    "wedge": ((0, 1, 2, 3), (1, 2, 4, 3), (2, 4, 5, 3)),
    "hexahedron": ((0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)),
}


@dataclass
class MeshSource:
    """meshio-like container: points, cell blocks, per-block physical tags, names."""
    points: np.ndarray
    cells: list            # [(type_name, int array (n, k))]
    physical: list         # [int array (n,)] aligned with cells
    field_data: dict       # name -> (tag, dim)
    periodic_map: np.ndarray | None = None


@dataclass
class Block:
    element_type: str
    connectivity: np.ndarray
    centers: np.ndarray
    volumes: np.ndarray
    geometry_connectivity: np.ndarray | None = None


@dataclass
class FaceBlock:
    face_type: str
    nodes: np.ndarray
    owner_block: np.ndarray
    owner_local: np.ndarray
    owner_face: np.ndarray
    neighbor_block: np.ndarray
    neighbor_local: np.ndarray
    neighbor_face: np.ndarray
    centers: np.ndarray
    normals: np.ndarray
    areas: np.ndarray
    boundary_tags: np.ndarray
    periodic: np.ndarray = field(default=None)

    @property
    def internal(self):
        return self.neighbor_block >= 0


def _tet_volume(v):
    return abs(np.linalg.det(np.stack([v[1] - v[0], v[2] - v[0], v[3] - v[0]], axis=1))) / 6.0


class Mesh:
    def __init__(self, source: MeshSource):
        self.points = np.asarray(source.points, np.float64)
        self.physical_names = {name: int(v[0]) for name, v in source.field_data.items()}
        self.canon = (np.arange(len(self.points)) if source.periodic_map is None
                      else np.asarray(source.periodic_map))
        self.element_blocks = self._blocks(source)
        tags = self._boundary_tags(source)
        self.face_blocks = self._faces(tags)
        self._validate()

    def _blocks(self, source):
        grouped = {}
        for (ctype, data) in source.cells:
            if ctype in ALIASES:
                grouped.setdefault(ALIASES[ctype][0], []).append((ctype, np.asarray(data, np.int64)))
        if not grouped:
            raise ValueError("Mesh contains no tetrahedron, wedge, or hexahedron")
        blocks = []
        for etype in ("hexahedron", "wedge", "tetra"):
            if etype not in grouped:
                continue
            ctype = grouped[etype][0][0]
            geometry = np.concatenate([a for _, a in grouped[etype]]).astype(np.int32)
            conn = geometry[:, :ALIASES[ctype][1]]
            gconn = geometry[:, P2_PERMUTATIONS[ctype]] if ctype in P2_PERMUTATIONS else None
            centers, volumes = [], []
            for cell in conn:
                v = self.points[cell]
                pieces = [v[list(t)] for t in TETRA_DECOMPOSITIONS[etype]]
                vols = [_tet_volume(p) for p in pieces]
                total = float(np.sum(vols))
                centers.append(np.sum([vol * p.mean(axis=0) for vol, p in zip(vols, pieces)], axis=0) / total)
                volumes.append(total)
            blocks.append(Block(etype, conn, np.asarray(centers), np.asarray(volumes), gconn))
        return blocks

    def _boundary_tags(self, source):
        tags = {}
        for (ctype, data), phys in zip(source.cells, source.physical):
            n = 3 if ctype == "triangle" else (4 if ctype == "quad" else None)
            if n is None:
                continue
            for nodes, tag in zip(np.asarray(data)[:, :n], np.asarray(phys)):
                key = tuple(sorted(int(self.canon[v]) for v in nodes))
                if key in tags and tags[key] != int(tag):
                    raise ValueError(f"Conflicting physical tags on face {key}")
                tags[key] = int(tag)
        return tags

    def _face_geometry(self, nodes, owner_center):
        v = self.points[nodes]
        center = v.mean(axis=0)
        if len(nodes) == 3:
            area_vector = 0.5 * np.cross(v[1] - v[0], v[2] - v[0])
        else:
            area_vector = 0.5 * (np.cross(v[1] - v[0], v[2] - v[0]) + np.cross(v[2] - v[0], v[3] - v[0]))
        if np.dot(area_vector, center - owner_center) < 0.0:
            area_vector = -area_vector
        area = np.linalg.norm(area_vector)
        return center, area_vector / area, area

    def _faces(self, boundary_tags):
        pending = {}
        finished = {"triangle": [], "quad": []}
        for b, block in enumerate(self.element_blocks):
            for e, cell in enumerate(block.connectivity):
                for lf, loc in enumerate(LOCAL_FACES[block.element_type]):
                    nodes = np.asarray([cell[i] for i in loc], np.int32)
                    key = tuple(sorted(int(self.canon[v]) for v in nodes))
                    rec = (b, e, lf, nodes)
                    if key in pending:
                        finished["triangle" if len(nodes) == 3 else "quad"].append((pending.pop(key), rec, -1))
                    else:
                        pending[key] = rec
        for key, rec in pending.items():
            finished["triangle" if len(key) == 3 else "quad"].append((rec, None, boundary_tags.get(key, -1)))
        out = {}
        for ftype, records in finished.items():
            if not records:
                continue
            cols = {k: [] for k in ("nodes", "ob", "ol", "of", "nb", "nl", "nf", "c", "n", "a", "t", "p")}
            for owner, nbr, tag in records:
                ob, ol, of, nodes = owner
                center, normal, area = self._face_geometry(nodes, self.element_blocks[ob].centers[ol])
                periodic = False
                if nbr is None:
                    nb = nl = nf = -1
                else:
                    nb, nl, nf, nnodes = nbr
                    periodic = not np.array_equal(np.sort(nodes), np.sort(nnodes))
                    if not periodic:
                        disp = self.element_blocks[nb].centers[nl] - self.element_blocks[ob].centers[ol]
                        if np.dot(normal, disp) < 0.0:
                            normal = -normal
                for k, v in zip(cols, (nodes, ob, ol, of, nb, nl, nf, center, normal, area, tag, periodic)):
                    cols[k].append(v)
            out[ftype] = FaceBlock(
                ftype, np.asarray(cols["nodes"], np.int32), np.asarray(cols["ob"], np.int32),
                np.asarray(cols["ol"], np.int32), np.asarray(cols["of"], np.int32),
                np.asarray(cols["nb"], np.int32), np.asarray(cols["nl"], np.int32),
                np.asarray(cols["nf"], np.int32), np.asarray(cols["c"]), np.asarray(cols["n"]),
                np.asarray(cols["a"]), np.asarray(cols["t"], np.int32), np.asarray(cols["p"], bool))
        return out

    def _validate(self):
        vols = np.concatenate([b.volumes for b in self.element_blocks])
        if not np.all(np.isfinite(vols)) or np.any(vols <= 0.0):
            raise ValueError("Mesh contains non-positive or invalid cell volumes")
        for ftype, fb in self.face_blocks.items():
            if np.any(fb.areas <= 0.0):
                raise ValueError(f"Mesh contains invalid {ftype} face areas")
            if np.any(fb.boundary_tags[fb.internal] != -1):
                raise ValueError("Internal faces cannot have boundary tags")
            if np.any(fb.boundary_tags[~fb.internal] < 0):
                missing = int(np.sum(fb.boundary_tags[~fb.internal] < 0))
                raise ValueError(f"{missing} boundary {ftype} faces lack physical tags")
