"""Type-blocked hybrid mesh: element blocks and paired faces (vectorised).

Mirrors ``HybridMesh`` of superboss2300/jax-fluid-sim (``hybrid/mesh.py:178-507``):
element blocks are ordered hexahedron -> wedge -> tetra; a face's owner is
the first (block, cell, local face) in that visiting order; internal faces are
listed in the order their second visitor arrives, boundary faces afterwards in
first-visit order; the face normal comes from the owner's corners and points
toward the neighbour centre.  The pairing is one parallel sort of the visits by
(sorted corner key, visit) on the host cores (``dgb_pair_faces``) instead of a
Python dictionary walk, and reproduces the reference's face order exactly.

Periodicity (not in the reference): ``MeshSource.periodic_map`` gives each
point a canonical id used for face keys and neighbour alignment.
"""

from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _native
from .meshgen import MeshSource
from .reference import LOCAL_FACES

TET_SPLITS = {
    "tetra": ((0, 1, 2, 3),),
    "wedge": ((0, 1, 2, 3), (1, 2, 4, 3), (2, 4, 5, 3)),
    "hexahedron": ((0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)),
}
CORNER_COUNT = {"tetra": 4, "wedge": 6, "hexahedron": 8}
# Source cell types (meshio names) -> (element type, corner count); hybrid/mesh.py:11-20
ALIASES = {"tetra": ("tetra", 4), "tetra10": ("tetra", 4), "wedge": ("wedge", 6), "wedge15": ("wedge", 6),
           "wedge18": ("wedge", 6), "hexahedron": ("hexahedron", 8), "hexahedron20": ("hexahedron", 8),
           "hexahedron27": ("hexahedron", 8)}
# Complete second-order cells carry curved geometry: their nodes in meshio/VTK order go to the
# second-order reference element's node order (hybrid/mesh.py:22-35).
P2_PERMUTATIONS = {
    "tetra10": np.asarray([0, 1, 2, 3, 4, 6, 7, 5, 8, 9], np.int32),
    "wedge18": np.asarray([0, 1, 2, 6, 9, 7, 3, 4, 5, 12, 14, 13, 8, 10, 11, 15, 17, 16], np.int32),
    "hexahedron27": np.asarray([0, 1, 8, 3, 2, 10, 11, 9, 24, 4, 5, 12, 7, 6, 14, 15, 13, 25,
                                16, 17, 22, 19, 18, 23, 20, 21, 26], np.int32),
}


@dataclass
class ElementBlock:
    element_type: str
    connectivity: np.ndarray
    centers: np.ndarray
    volumes: np.ndarray
    global_ids: np.ndarray
    source_cell_type: str = ""
    geometry_connectivity: np.ndarray | None = None   # second-order geometry nodes (curved cells)

    @property
    def geometry_degree(self):
        return 1 if self.geometry_connectivity is None else 2


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
    neighbor_nodes: np.ndarray

    @property
    def internal(self):
        return self.neighbor_block >= 0


def _cell_geometry(points, etype, conn):
    v = points[conn]                                            # (E, k, 3)
    vols, cents = [], []
    for t in TET_SPLITS[etype]:
        a, b, c, d = (v[:, i] for i in t)
        vol = np.abs(np.linalg.det(np.stack([b - a, c - a, d - a], axis=2))) / 6.0
        vols.append(vol)
        cents.append(vol[:, None] * (a + b + c + d) / 4.0)
    total = np.sum(vols, axis=0)
    return np.sum(cents, axis=0) / total[:, None], total


class HybridMesh:
    def __init__(self, source):
        if isinstance(source, (str, Path)):
            from .gmsh import read_gmsh
            source = read_gmsh(source)
        self.source = source
        self.points = np.asarray(source.points, np.float64)
        self.physical_names = {name: int(v[0]) for name, v in source.field_data.items()}
        self.canon = (np.arange(len(self.points)) if source.periodic_map is None
                      else np.asarray(source.periodic_map, np.int64))
        self.element_blocks = self._blocks(source)
        self.number_of_cells = sum(len(b.connectivity) for b in self.element_blocks)
        self.face_blocks = self._faces(self._boundary_tags(source))
        self.number_of_internal_faces = sum(int(fb.internal.sum()) for fb in self.face_blocks.values())
        self.number_of_boundary_faces = sum(int((~fb.internal).sum()) for fb in self.face_blocks.values())
        self._validate()

    def _blocks(self, source):
        """hybrid/mesh.py:238-286; one source cell type per element type (the reference would
        make two blocks of one element type, which the type-keyed state dicts cannot hold)."""
        grouped = {}
        for ctype, data in source.cells:
            if ctype in ALIASES:
                etype = ALIASES[ctype][0]
                if etype in grouped and grouped[etype][0] != ctype:
                    raise NotImplementedError(f"{etype} cells of two source types ({grouped[etype][0]}, {ctype})")
                grouped.setdefault(etype, (ctype, []))[1].append(np.asarray(data))
        if not grouped:
            raise ValueError("Mesh contains no tetrahedron, wedge, or hexahedron")
        blocks, start = [], 0
        for etype in ("hexahedron", "wedge", "tetra"):
            if etype in grouped:
                ctype, arrays = grouped[etype]
                geometry = np.concatenate(arrays).astype(np.int32)
                conn = np.ascontiguousarray(geometry[:, :ALIASES[ctype][1]])
                c, v = _cell_geometry(self.points, etype, conn)
                gconn = (np.ascontiguousarray(geometry[:, P2_PERMUTATIONS[ctype]])
                         if ctype in P2_PERMUTATIONS else None)
                blocks.append(ElementBlock(etype, conn, c, v, np.arange(start, start + len(conn), dtype=np.int32),
                                           ctype, gconn))
                start += len(conn)
        return blocks

    def geometry(self, block):
        """(geometry reference element, node coordinates (E, n, 3)) of a block: the second-order
        map of curved cells, the first-order map otherwise (hybrid/geometry.py:102-110)."""
        from .reference import RefElement
        cache = self.__dict__.setdefault("_geometry", {})
        key = id(block)
        if key not in cache:
            if block.geometry_connectivity is not None:
                cache[key] = (block, RefElement(block.element_type, 2), self.points[block.geometry_connectivity])
            else:
                cache[key] = (block, RefElement(block.element_type, 1), self.points[block.connectivity])
        return cache[key][1], cache[key][2]

    def _boundary_tags(self, source):
        keys, tags = [], []
        for (ctype, data), phys in zip(source.cells, source.physical):
            k = 3 if ctype == "triangle" else (4 if ctype == "quad" else 0)
            if k:
                nodes = np.sort(self.canon[np.asarray(data)[:, :k]], axis=1)
                keys.append(nodes)
                tags.append(np.asarray(phys, np.int64))
        table = {}
        for nodes, t in zip(keys, tags):
            for key, tag in zip(map(tuple, nodes.tolist()), t.tolist()):
                if table.get(key, tag) != tag:
                    raise ValueError(f"Conflicting physical tags on face {key}")
                table[key] = tag
        return table

    def _faces(self, boundary_tags):
        # every (block, cell, local face) visit in the reference's order
        recs = {3: [], 4: []}
        order = 0
        for b, block in enumerate(self.element_blocks):
            E = len(block.connectivity)
            for lf, loc in enumerate(LOCAL_FACES[block.element_type]):
                nodes = block.connectivity[:, list(loc)]
                visit = order + np.arange(E) * len(LOCAL_FACES[block.element_type]) + lf
                recs[len(loc)].append((np.full(E, b), np.arange(E), np.full(E, lf), nodes, visit))
            order += E * len(LOCAL_FACES[block.element_type])
        out = {}
        for k, ftype in ((3, "triangle"), (4, "quad")):
            if not recs[k]:
                continue
            blk, loc, lface, nodes, visit = (np.concatenate([r[i] for r in recs[k]]) for i in range(5))
            key = np.sort(self.canon[nodes], axis=1)
            # pairs equal keys; faces in the reference's order (host threads)
            own, nbr = _native.pair_faces(key, visit)
            has_n = nbr >= 0
            nbr_c = np.where(has_n, nbr, 0)
            fnodes = nodes[own]
            tags = np.full(len(own), -1, np.int32)
            bkeys = key[own[~has_n]]
            tags[~has_n] = [boundary_tags.get(tuple(r), -1) for r in bkeys.tolist()]
            ob, ol = blk[own].astype(np.int32), loc[own].astype(np.int32)
            all_centers = np.concatenate([b.centers for b in self.element_blocks])
            offsets = np.cumsum([0] + [len(b.connectivity) for b in self.element_blocks])
            owner_center = all_centers[offsets[ob] + ol]
            center, normal, area = self._face_geometry(fnodes, owner_center)
            nb = np.where(has_n, blk[nbr_c], -1).astype(np.int32)
            nl = np.where(has_n, loc[nbr_c], -1).astype(np.int32)
            nf = np.where(has_n, lface[nbr_c], -1).astype(np.int32)
            nnodes = np.where(has_n[:, None], nodes[nbr_c], -1).astype(np.int32)
            periodic = has_n & np.any(np.sort(fnodes, axis=1) != np.sort(nnodes, axis=1), axis=1)
            flip_check = has_n & ~periodic
            if np.any(flip_check):
                idx = np.flatnonzero(flip_check)
                nc = all_centers[offsets[nb[idx]] + nl[idx]]
                disp = nc - owner_center[idx]
                flip = np.sum(normal[idx] * disp, axis=1) < 0.0
                normal[idx[flip]] *= -1.0
            out[ftype] = FaceBlock(ftype, fnodes.astype(np.int32), ob, ol, lface[own].astype(np.int32), nb, nl, nf,
                                   center, normal, area, tags, nnodes)
        return out

    def _face_geometry(self, nodes, owner_center):
        v = self.points[nodes]
        center = v.mean(axis=1)
        if nodes.shape[1] == 3:
            av = 0.5 * np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
        else:
            av = 0.5 * (np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]) + np.cross(v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]))
        flip = np.sum(av * (center - owner_center), axis=1) < 0.0
        av[flip] *= -1.0
        area = np.linalg.norm(av, axis=1)
        return center, av / area[:, None], area

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
