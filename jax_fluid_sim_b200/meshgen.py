"""Seeded synthetic meshes for the benchmark workloads and the parity tests.

The reference ships Gmsh files made by gmsh/meshio tools that are not usable
here; these numpy generators produce first-order meshes of the same kinds:

* ``box_hex``       jittered (or uniform) structured hex box, optional periodicity
                    (Taylor-Green cube, vortex cube);
* ``smoke_mesh``    one hex + one wedge + one tet sharing a quad and a triangle
                    (same cells as the reference's ``tools/generate_hybrid_smoke_mesh.py:15-86``);
* ``mixed_block``   a conforming 2x1x2 block of hex / z-prisms / x-prisms / Kuhn tets;
* ``sphere_oh_grid`` body-fitted O/H hex grid around a sphere in a box
                    (cubed-sphere O-grid inside, H-grid outside).

All return a :class:`MeshSource` (meshio-like: points, cell blocks, physical
tags per block, physical names, optional periodic point map).
"""

from dataclasses import dataclass

import numpy as np

HEX_FACES = ((0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7))
WEDGE_FACES = ((0, 2, 1), (3, 4, 5), (0, 1, 4, 3), (1, 2, 5, 4), (2, 0, 3, 5))
TET_FACES = ((0, 2, 1), (0, 1, 3), (1, 2, 3), (2, 0, 3))
FACES = {"hexahedron": HEX_FACES, "wedge": WEDGE_FACES, "tetra": TET_FACES}


@dataclass
class MeshSource:
    points: np.ndarray
    cells: list            # [(type_name, (n, k) int array)]
    physical: list         # [(n,) int array] aligned with cells
    field_data: dict       # name -> (tag, dim)
    periodic_map: np.ndarray | None = None

    def save(self, path, **extra):
        arrays = {"points": self.points, "cell_types": np.asarray([c[0] for c in self.cells])}
        for i, ((_, conn), phys) in enumerate(zip(self.cells, self.physical)):
            arrays[f"cell_conn_{i}"] = np.asarray(conn, np.int32)
            arrays[f"cell_phys_{i}"] = np.asarray(phys, np.int32)
        names = list(self.field_data)
        arrays["field_names"] = np.asarray(names)
        arrays["field_tags"] = np.asarray([self.field_data[n][0] for n in names], np.int32)
        arrays["field_dims"] = np.asarray([self.field_data[n][1] for n in names], np.int32)
        if self.periodic_map is not None:
            arrays["periodic_map"] = np.asarray(self.periodic_map, np.int64)
        arrays.update(extra)
        np.savez_compressed(path, **arrays)

    @staticmethod
    def from_arrays(arrays):
        types = [str(t) for t in arrays["cell_types"]]
        cells = [(t, np.asarray(arrays[f"cell_conn_{i}"])) for i, t in enumerate(types)]
        phys = [np.asarray(arrays[f"cell_phys_{i}"]) for i in range(len(types))]
        fd = {str(n): (int(t), int(d)) for n, t, d in zip(arrays["field_names"], arrays["field_tags"],
                                                          arrays["field_dims"])}
        pm = np.asarray(arrays["periodic_map"]) if "periodic_map" in arrays else None
        return MeshSource(np.asarray(arrays["points"], np.float64), cells, phys, fd, pm)


def _boundary_cells(volume_cells, canon, tagger):
    """Unpaired faces (by canonical sorted key) become boundary tri/quad cells."""
    seen = {}
    for ctype, conn in volume_cells:
        for cell in conn:
            for loc in FACES[ctype]:
                nodes = tuple(int(cell[i]) for i in loc)
                key = tuple(sorted(int(canon[v]) for v in nodes))
                seen.setdefault(key, []).append(nodes)
    tris, quads, ttag, qtag = [], [], [], []
    for recs in seen.values():
        if len(recs) != 1:
            continue
        nodes = recs[0]
        tag = tagger(np.asarray(nodes))
        if len(nodes) == 3:
            tris.append(nodes)
            ttag.append(tag)
        else:
            quads.append(nodes)
            qtag.append(tag)
    out, phys = [], []
    if tris:
        out.append(("triangle", np.asarray(tris, np.int32)))
        phys.append(np.asarray(ttag, np.int32))
    if quads:
        out.append(("quad", np.asarray(quads, np.int32)))
        phys.append(np.asarray(qtag, np.int32))
    return out, phys


def _box_tagger(points, lo, hi, names):
    """Tag a boundary face by the box plane its centre lies on."""
    def tag(nodes):
        c = points[nodes].mean(axis=0)
        scale = np.max(hi - lo)
        for axis in range(3):
            if abs(c[axis] - lo[axis]) < 1e-9 * scale:
                return names[axis][0]
            if abs(c[axis] - hi[axis]) < 1e-9 * scale:
                return names[axis][1]
        return names[3]
    return tag


def box_hex(n=(4, 4, 4), lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), jitter=0.0, seed=0,
            periodic=(False, False, False),
            plane_tags=(("inlet", "outlet"), ("walls", "walls"), ("sphere_wall", "sphere_wall"))):
    """Structured hex box; interior vertex columns jittered by +-jitter*h in x, y (seeded).

    Periodic axes identify the lo and hi planes through ``periodic_map`` (vertices
    on those planes are not jittered in that axis so the planes stay congruent).
    """
    nx, ny, nz = n
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    axes = [np.linspace(lo[d], hi[d], n[d] + 1) for d in range(3)]
    Z, Y, X = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    points = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

    def pid(i, j, k):
        return (k * (ny + 1) + j) * (nx + 1) + i

    K, J, I = (a.ravel() for a in np.indices((nz + 1, ny + 1, nx + 1)))
    idx = np.stack([I, J, K], axis=1)          # row r describes point r
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        h = (hi - lo) / np.asarray(n)
        # one (dx, dy) per vertical column of vertices, none in z: cells stay
        # non-affine but keep planar faces, so the reference's check of the
        # mapped volume against the tetrahedral-split volume (rtol 1e-4) holds
        column = rng.uniform(-jitter, jitter, size=((ny + 1) * (nx + 1), 2))
        delta = np.zeros((len(idx), 3))
        delta[:, :2] = column[idx[:, 1] * (nx + 1) + idx[:, 0]] * h[None, :2]
        for d in range(3):
            # a vertex on a box face may slide within the face but not leave it
            delta[(idx[:, d] == 0) | (idx[:, d] == n[d]), d] = 0.0
        for d in range(3):
            if periodic[d]:
                # periodic partner planes stay congruent: hi-plane vertices copy their lo partners
                hi_side = np.flatnonzero(idx[:, d] == n[d])
                partner = idx[hi_side].copy()
                partner[:, d] = 0
                delta[hi_side] = delta[pid(partner[:, 0], partner[:, 1], partner[:, 2])]
        points = points + delta
    conn = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                conn.append([pid(i, j, k), pid(i + 1, j, k), pid(i + 1, j + 1, k), pid(i, j + 1, k),
                             pid(i, j, k + 1), pid(i + 1, j, k + 1), pid(i + 1, j + 1, k + 1), pid(i, j + 1, k + 1)])
    conn = np.asarray(conn, np.int32)
    canon = np.arange(len(points))
    if any(periodic):
        ci = np.where(periodic[0] & (I == nx), 0, I)
        cj = np.where(periodic[1] & (J == ny), 0, J)
        ck = np.where(periodic[2] & (K == nz), 0, K)
        canon = np.empty(len(points), np.int64)
        canon[pid(I, J, K)] = pid(ci, cj, ck)
    names = sorted({n for pair in plane_tags for n in pair})
    field = {"fluid": (1, 3)}
    for t, name in enumerate(names):
        field[name] = (10 + t, 2)
    tag_of = {name: field[name][0] for name in names}
    tagger = _box_tagger(points, lo, hi, [(tag_of[a], tag_of[b]) for a, b in plane_tags] + [0])
    vol = [("hexahedron", conn)]
    bcells, bphys = _boundary_cells(vol, canon, tagger)
    used = {int(t) for p in bphys for t in p}
    field = {k: v for k, v in field.items() if k == "fluid" or v[0] in used}
    return MeshSource(points, vol + bcells, [np.ones(len(conn), np.int32)] + bphys, field,
                      canon if any(periodic) else None)


def smoke_mesh():
    """One hex, one wedge, one tet; all boundary faces tagged 'walls' (13)."""
    points = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [0, 1, 1], [0, 0, 2],
                       [1, -1, 0], [0, -1, 0], [1, -1, 1], [0, -1, 1]], float)
    vol = [("hexahedron", np.array([[0, 1, 7, 8, 3, 4, 9, 10]], np.int32)),
           ("wedge", np.array([[0, 1, 2, 3, 4, 5]], np.int32)),
           ("tetra", np.array([[3, 4, 5, 6]], np.int32))]
    bcells, bphys = _boundary_cells(vol, np.arange(len(points)), lambda nodes: 13)
    return MeshSource(points, vol + bcells, [np.ones(1, np.int32)] * 3 + bphys,
                      {"fluid": (1, 3), "walls": (13, 2)})


def _kuhn_tets(c):
    """Six tetrahedra of the unit-cube corner array c[ix][iy][iz] sharing the main diagonal."""
    out = []
    for a, b in ((0, 1), (0, 2), (1, 0), (1, 2), (2, 0), (2, 1)):
        e = [0, 0, 0]
        path = [tuple(e)]
        for axis in (a, b, 3 - a - b):
            e[axis] = 1
            path.append(tuple(e))
        out.append([c[p] for p in path])
    return out


def mixed_block(jitter=0.1, seed=0):
    """2x1x2 cubes: hex | z-prisms (bottom row), x-prisms | Kuhn tets (top row)."""
    n = (2, 1, 2)
    grid = np.stack(np.meshgrid(np.arange(3), np.arange(2), np.arange(3), indexing="ij"), -1).reshape(-1, 3)
    points = grid.astype(float)
    index = {tuple(p): i for i, p in enumerate(grid)}
    rng = np.random.default_rng(seed)
    column = rng.uniform(-jitter, jitter, size=(3, 2, 2))      # (x, y) shift per vertex column
    for i, p in enumerate(grid):
        inner = np.asarray([(0 < p[d] < n[d]) for d in range(2)], float)
        points[i, :2] += column[p[0], p[1]] * inner

    def corners(i0, j0, k0):
        return {(a, b, c): index[(i0 + a, j0 + b, k0 + c)] for a in (0, 1) for b in (0, 1) for c in (0, 1)}

    hexes, wedges, tets = [], [], []
    c = corners(0, 0, 0)
    hexes.append([c[0, 0, 0], c[1, 0, 0], c[1, 1, 0], c[0, 1, 0], c[0, 0, 1], c[1, 0, 1], c[1, 1, 1], c[0, 1, 1]])
    c = corners(1, 0, 0)    # prisms extruded along z, triangles split by the (0,0)-(1,1) xy diagonal
    wedges.append([c[0, 0, 0], c[1, 0, 0], c[1, 1, 0], c[0, 0, 1], c[1, 0, 1], c[1, 1, 1]])
    wedges.append([c[0, 0, 0], c[1, 1, 0], c[0, 1, 0], c[0, 0, 1], c[1, 1, 1], c[0, 1, 1]])
    c = corners(0, 0, 1)    # prisms extruded along x, triangles split by the (0,0)-(1,1) yz diagonal
    wedges.append([c[0, 0, 0], c[0, 1, 0], c[0, 1, 1], c[1, 0, 0], c[1, 1, 0], c[1, 1, 1]])
    wedges.append([c[0, 0, 0], c[0, 1, 1], c[0, 0, 1], c[1, 0, 0], c[1, 1, 1], c[1, 0, 1]])
    tets.extend(_kuhn_tets(corners(1, 0, 1)))
    vol = [("hexahedron", np.asarray(hexes, np.int32)), ("wedge", np.asarray(wedges, np.int32)),
           ("tetra", np.asarray(tets, np.int32))]
    field = {"fluid": (1, 3), "inlet": (10, 2), "outlet": (11, 2), "walls": (12, 2)}
    tagger = _box_tagger(points, np.zeros(3), np.asarray(n, float), [(10, 11), (12, 12), (12, 12), 12])
    bcells, bphys = _boundary_cells(vol, np.arange(len(points)), tagger)
    phys = [np.ones(len(v[1]), np.int32) for v in vol]
    return MeshSource(points, vol + bcells, phys + bphys, field)


def hybrid_box(n=(8, 8, 8), lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), jitter=0.1, seed=0, fill=2.0 / 3.0):
    """Fully periodic, conforming box of n cubes, each one hexahedron, two prisms or six tetrahedra.

    The reference pairs faces by their vertex sets only (hybrid/mesh.py:391-405), so a quad
    may only meet a quad and a triangle a triangle with the same diagonal.  Every triangulated
    cube face here is cut along the diagonal through the cube's (0,0,0)-(1,1,1) corners, and a
    cube's two faces normal to axis d are triangulated together or not at all, by a flag that
    must then be the same along the whole line of cubes in d.  Three seeded 0/1 sequences a(i),
    b(j), c(k), each with round(fill * n) ones, set the flags (x: b and c, y: a and c, z: a and b):
    all three set gives six Kuhn tetrahedra round the main diagonal, one set gives two prisms
    extruded along that axis, none a hexahedron.  fill = 2/3 puts roughly a third of the cubes in
    each kind; the counts are in ``hybrid_box_fractions``.  Vertex columns are jittered by up to
    jitter*h in x and y (seeded, periodic partners together), which keeps every face planar.
    The lo/hi planes are identified in all three directions, so at least 3 cubes per direction
    are needed for faces to be told apart by their vertex sets.
    """
    nx, ny, nz = n
    if min(n) < 3:
        raise ValueError("hybrid_box needs at least 3 cubes per direction")
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    h = (hi - lo) / np.asarray(n, float)
    K, J, I = (a.ravel() for a in np.indices((nz + 1, ny + 1, nx + 1)))
    points = lo + np.stack([I, J, K], axis=1) * h

    def pid(i, j, k):
        return (k * (ny + 1) + j) * (nx + 1) + i

    rng = np.random.default_rng(seed)

    def flags(m):
        f = np.zeros(m, bool)
        f[:int(round(fill * m))] = True
        return rng.permutation(f)

    a, b, c = flags(nx), flags(ny), flags(nz)
    if jitter > 0.0:
        column = rng.uniform(-jitter, jitter, size=(ny + 1, nx + 1, 2))
        column[-1, :] = column[0, :]
        column[:, -1] = column[:, 0]
        points[:, :2] += column[J, I] * h[:2]
    canon = pid(np.where(I == nx, 0, I), np.where(J == ny, 0, J), np.where(K == nz, 0, K)).astype(np.int64)
    hexes, wedges, tets = [], [], []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                q = {(x, y, z): pid(i + x, j + y, k + z) for x in (0, 1) for y in (0, 1) for z in (0, 1)}
                tx, ty, tz = b[j] and c[k], a[i] and c[k], a[i] and b[j]
                if tx and ty and tz:     # odd axis orders (1, 2, 5) are left-handed: swap two nodes
                    tets.extend([t[0], t[2], t[1], t[3]] if r in (1, 2, 5) else t
                                for r, t in enumerate(_kuhn_tets(q)))
                elif tz:              # triangles in the z-faces, right-handed about +z
                    wedges.append([q[0, 0, 0], q[1, 0, 0], q[1, 1, 0], q[0, 0, 1], q[1, 0, 1], q[1, 1, 1]])
                    wedges.append([q[0, 0, 0], q[1, 1, 0], q[0, 1, 0], q[0, 0, 1], q[1, 1, 1], q[0, 1, 1]])
                elif tx:              # about +x
                    wedges.append([q[0, 0, 0], q[0, 1, 0], q[0, 1, 1], q[1, 0, 0], q[1, 1, 0], q[1, 1, 1]])
                    wedges.append([q[0, 0, 0], q[0, 1, 1], q[0, 0, 1], q[1, 0, 0], q[1, 1, 1], q[1, 0, 1]])
                elif ty:              # about +y
                    wedges.append([q[0, 0, 0], q[0, 0, 1], q[1, 0, 1], q[0, 1, 0], q[0, 1, 1], q[1, 1, 1]])
                    wedges.append([q[0, 0, 0], q[1, 0, 1], q[1, 0, 0], q[0, 1, 0], q[1, 1, 1], q[1, 1, 0]])
                else:
                    hexes.append([q[0, 0, 0], q[1, 0, 0], q[1, 1, 0], q[0, 1, 0],
                                  q[0, 0, 1], q[1, 0, 1], q[1, 1, 1], q[0, 1, 1]])
    vol = [(name, np.asarray(conn, np.int32)) for name, conn in
           (("hexahedron", hexes), ("wedge", wedges), ("tetra", tets)) if conn]
    return MeshSource(points, vol, [np.ones(len(v[1]), np.int32) for v in vol], {"fluid": (1, 3)}, canon)


def hybrid_box_fractions(source):
    """Fractions of cubes split into hexahedra, prism pairs and six tetrahedra."""
    counts = {name: len(conn) for name, conn in source.cells}
    cubes = np.array([counts.get("hexahedron", 0), counts.get("wedge", 0) / 2, counts.get("tetra", 0) / 6])
    return dict(zip(("hexahedron", "wedge", "tetra"), cubes / cubes.sum()))


def sphere_oh_grid(radius=0.5, box=((-4.0, 12.0), (-6.0, 6.0), (-6.0, 6.0)), cube=1.5, n=24, n_radial=20,
                   outer=((8, 32), (12, 12), (12, 12)), clustering=1.6):
    """Body-fitted O/H hex grid around a sphere centred at the origin.

    A structured H-grid fills the box outside the cube [-cube, cube]^3 (n cells per cube
    edge); inside, n_radial layers of an O-grid connect the cube's surface grid to the
    sphere, each surface node moving along the straight line from its projection on the
    sphere (layer spacing clustered toward the wall by ``clustering``).  Tags: inlet
    (x min), outlet (x max), walls (y and z planes, slip), sphere_wall (no-slip body).
    """
    segs = []
    for d in range(3):
        lo, hi = box[d]
        segs.append(np.concatenate([np.linspace(lo, -cube, outer[d][0] + 1),
                                    np.linspace(-cube, cube, n + 1)[1:],
                                    np.linspace(cube, hi, outer[d][1] + 1)[1:]]))
    nxn, nyn, nzn = (len(s) for s in segs)
    Z, Y, X = np.meshgrid(segs[2], segs[1], segs[0], indexing="ij")
    points = [np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)]

    def bid(i, j, k):
        return (k * nyn + j) * nxn + i

    c0 = (outer[0][0], outer[1][0], outer[2][0])
    inside = lambda i, j, k: (c0[0] <= i < c0[0] + n) and (c0[1] <= j < c0[1] + n) and (c0[2] <= k < c0[2] + n)
    hexes = []
    for k in range(nzn - 1):
        for j in range(nyn - 1):
            for i in range(nxn - 1):
                if inside(i, j, k):
                    continue
                hexes.append([bid(i, j, k), bid(i + 1, j, k), bid(i + 1, j + 1, k), bid(i, j + 1, k),
                              bid(i, j, k + 1), bid(i + 1, j, k + 1), bid(i + 1, j + 1, k + 1), bid(i, j + 1, k + 1)])
    # O-grid nodes: one radial line per cube-surface node
    base = points[0]
    line_of = {}
    next_id = len(base)
    extra = []
    s = (np.arange(n_radial) / n_radial) ** clustering          # layer l fraction toward the cube
    rng_ = range(n + 1)
    for a in rng_:
        for b in rng_:
            for c in rng_:
                if 0 < a < n and 0 < b < n and 0 < c < n:
                    continue
                node = bid(c0[0] + a, c0[1] + b, c0[2] + c)
                p = base[node]
                q = radius * p / np.linalg.norm(p)
                ids = []
                for l in range(n_radial):
                    extra.append((1.0 - s[l]) * q + s[l] * p)
                    ids.append(next_id)
                    next_id += 1
                ids.append(node)
                line_of[(a, b, c)] = ids
    points.append(np.asarray(extra))
    points = np.concatenate(points)
    # six cube faces: (fixed axis, value), in-plane axes
    wall_quads = []
    for axis in range(3):
        for val in (0, n):
            u_ax, v_ax = [d for d in range(3) if d != axis]
            for u in range(n):
                for v in range(n):
                    def key(du, dv):
                        idx = [0, 0, 0]
                        idx[axis] = val
                        idx[u_ax] = u + du
                        idx[v_ax] = v + dv
                        return tuple(idx)
                    quad = [line_of[key(0, 0)], line_of[key(1, 0)], line_of[key(1, 1)], line_of[key(0, 1)]]
                    for l in range(n_radial):
                        cell = [quad[m][l] for m in range(4)] + [quad[m][l + 1] for m in range(4)]
                        hexes.append(cell)
                    wall_quads.append([quad[m][0] for m in range(4)])
    hexes = np.asarray(hexes, np.int64)
    # positive orientation: swap the two quads of any inverted cell
    v = points[hexes]
    det = np.einsum("ij,ij->i", np.cross(v[:, 1] - v[:, 0], v[:, 3] - v[:, 0]), v[:, 4] - v[:, 0])
    flip = det < 0
    hexes[flip] = hexes[flip][:, [4, 5, 6, 7, 0, 1, 2, 3]]
    field = {"fluid": (1, 3), "inlet": (10, 2), "outlet": (11, 2), "walls": (12, 2), "sphere_wall": (13, 2)}
    lo = np.asarray([b[0] for b in box])
    hi = np.asarray([b[1] for b in box])
    tagger = _box_tagger(points, lo, hi, [(10, 11), (12, 12), (12, 12), 13])
    vol = [("hexahedron", hexes.astype(np.int32))]
    bcells, bphys = _boundary_cells_fast(vol, points, tagger)
    return MeshSource(points, vol + bcells, [np.ones(len(hexes), np.int32)] + bphys, field)


def curved_box(n=(3, 3, 2), lo=(0.0, 0.0, 0.0), hi=(1.5, 1.5, 1.0), amplitude=0.05,
               plane_tags=(("inlet", "outlet"), ("walls", "walls"), ("sphere_wall", "sphere_wall"))):
    """Box of curved triquadratic hexahedra ("hexahedron27" cells, node order as meshio gives
    it, which the mesh maps to the second-order reference element's order).

    The nodes of a (2n+1)^3 grid at half spacing are displaced by amplitude * h * S(x) along
    (1, 1, 1), S = prod_d sin(pi (x_d - lo_d) / L_d), which vanishes on the box faces: interior
    faces and cells curve while the boundary stays on the box planes.  Boundary quadrilaterals
    are tagged per plane as in ``box_hex``."""
    from .reference import RefElement
    from .mesh import P2_PERMUTATIONS
    nx, ny, nz = n
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    L = hi - lo
    h = L / np.asarray(n, float)
    axes = [np.linspace(lo[d], hi[d], 2 * n[d] + 1) for d in range(3)]
    Z, Y, X = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    points = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    bump = np.prod(np.sin(np.pi * (points - lo) / L), axis=1)
    points = points + amplitude * np.min(h) * bump[:, None] * np.ones(3)

    def gid(i, j, k):
        return (k * (2 * ny + 1) + j) * (2 * nx + 1) + i

    offsets = np.rint(2.0 * RefElement("hexahedron", 2).nodes).astype(int)     # internal order, (27, 3)
    perm = P2_PERMUTATIONS["hexahedron27"]
    cells27, corners = [], []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                internal = [gid(2 * i + a, 2 * j + b, 2 * k + c) for a, b, c in offsets]
                meshio_order = np.empty(27, np.int64)
                meshio_order[perm] = internal
                cells27.append(meshio_order)
                corners.append(meshio_order[:8])
    cells27 = np.asarray(cells27, np.int32)
    corners = np.asarray(corners, np.int32)
    names = sorted({nm for pair in plane_tags for nm in pair})
    field = {"fluid": (1, 3)}
    for t, name in enumerate(names):
        field[name] = (10 + t, 2)
    tag_of = {name: field[name][0] for name in names}
    tagger = _box_tagger(points, lo, hi, [(tag_of[a], tag_of[b]) for a, b in plane_tags] + [0])
    bcells, bphys = _boundary_cells([("hexahedron", corners)], np.arange(len(points)), tagger)
    used = {int(t) for p in bphys for t in p}
    field = {k: v for k, v in field.items() if k == "fluid" or v[0] in used}
    return MeshSource(points, [("hexahedron27", cells27)] + bcells, [np.ones(len(cells27), np.int32)] + bphys, field)


def cylinder_o_grid(n_theta=96, n_radial=48, radius=0.5, outer_radius=15.0, span=1.0, growth=None):
    """Extruded O-grid around a cylinder of the given radius (axis z), one element deep.

    n_theta cells around, n_radial cells out to ``outer_radius`` with radii in geometric
    progression (ratio ``growth``, by default the one that keeps the wall cells square).
    Tags: cylinder_wall (no-slip body), inlet (outer faces whose centre has x < 0: far-field
    state), outlet (outer faces with x >= 0: copy), symmetry (the two span planes, slip).  With
    one element in the span a z-periodic pair of planes would make every side face's vertex set
    degenerate for the reference's vertex-key face pairing (hybrid/mesh.py:391-405); slip planes
    give the same residual for the span-invariant flow (w = 0, no z-gradients).
    """
    if growth is None:
        growth = (outer_radius / radius) ** (1.0 / n_radial)
    r = radius * growth ** np.arange(n_radial + 1)
    r = radius + (r - radius) * (outer_radius - radius) / (r[-1] - radius)
    th = 2.0 * np.pi * np.arange(n_theta) / n_theta
    K, J, I = (a.ravel() for a in np.indices((2, n_radial + 1, n_theta)))
    points = np.stack([r[J] * np.cos(th[I]), r[J] * np.sin(th[I]), span * K], axis=1)

    def pid(i, j, k):
        return (k * (n_radial + 1) + j) * n_theta + (i % n_theta)

    i, j = (a.ravel() for a in np.meshgrid(np.arange(n_theta), np.arange(n_radial), indexing="ij"))
    # counter-clockwise about +z: (i, j) -> (i, j+1) -> (i+1, j+1) -> (i+1, j)
    bottom = [pid(i, j, 0), pid(i, j + 1, 0), pid(i + 1, j + 1, 0), pid(i + 1, j, 0)]
    hexes = np.stack(bottom + [b + n_theta * (n_radial + 1) for b in bottom], axis=1).astype(np.int32)
    it = np.arange(n_theta)
    wall = np.stack([pid(it, 0, 0), pid(it + 1, 0, 0), pid(it + 1, 0, 1), pid(it, 0, 1)], axis=1)
    outer = np.stack([pid(it, n_radial, 0), pid(it, n_radial, 1), pid(it + 1, n_radial, 1),
                      pid(it + 1, n_radial, 0)], axis=1)
    ends = np.concatenate([hexes[:, :4], hexes[:, 4:]])
    xc = points[outer].mean(axis=1)[:, 0]
    field = {"fluid": (1, 3), "inlet": (10, 2), "outlet": (11, 2), "symmetry": (12, 2), "cylinder_wall": (13, 2)}
    quads = np.concatenate([wall, outer, ends]).astype(np.int32)
    tags = np.concatenate([np.full(n_theta, 13), np.where(xc < 0.0, 10, 11), np.full(len(ends), 12)]).astype(np.int32)
    return MeshSource(points, [("hexahedron", hexes), ("quad", quads)], [np.ones(len(hexes), np.int32), tags], field)


def union(sources):
    """Disjoint union of meshes with the same physical names: (MeshSource, counts) where
    counts[c][type] is the number of volume cells of each type that case c contributes; within
    each volume type the union lists case 0's cells first, then case 1's, and so on."""
    points, pmaps, offset = [], [], 0
    by_type, phys_by_type, counts = {}, {}, []
    field = dict(sources[0].field_data)
    for src in sources:
        if dict(src.field_data) != field:
            raise ValueError("union needs the same physical names and tags in every mesh")
        points.append(src.points)
        pmaps.append((np.arange(len(src.points)) if src.periodic_map is None else np.asarray(src.periodic_map))
                     + offset)
        count = {}
        for (ctype, conn), phys in zip(src.cells, src.physical):
            by_type.setdefault(ctype, []).append(np.asarray(conn) + offset)
            phys_by_type.setdefault(ctype, []).append(np.asarray(phys))
            count[ctype] = count.get(ctype, 0) + len(conn)
        counts.append(count)
        offset += len(src.points)
    cells = [(t, np.concatenate(c).astype(np.int32)) for t, c in by_type.items()]
    phys = [np.concatenate(phys_by_type[t]).astype(np.int32) for t in by_type]
    periodic = any(s.periodic_map is not None for s in sources)
    return MeshSource(np.concatenate(points), cells, phys, field, np.concatenate(pmaps) if periodic else None), counts


def _boundary_cells_fast(volume_cells, points, tagger):
    """Vectorised unpaired-face search for large hex meshes (same result as _boundary_cells)."""
    ctype, conn = volume_cells[0]
    faces = np.concatenate([conn[:, list(loc)] for loc in FACES[ctype]])
    key = np.sort(faces, axis=1)
    _, inv, counts = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    single = counts[inv.ravel()] == 1
    bq = faces[single]
    tags = np.asarray([tagger(q) for q in bq], np.int32)
    return [("quad", bq.astype(np.int32))], [tags]
