"""Host-side construction of the device plan (all tables the kernels read).

Geometry follows the reference's isoparametric mapping (``hybrid/geometry.py:139-362``;
first order, or second order for curved cells): per element and volume point the inverse
Jacobian and w|det J|; per element the dense inverse mass matrix with the sliver scale
``min(1, V/1e-4)``; per face and face point the unit normal and w*dA from the owner mapping; per face side the reference points (owner:
its local-face corners, neighbour: corners matched by node id), from which a
small set of distinct "trace codes" per element type is built.  Each code owns
a trace matrix (basis at the side's face points) and its reference-gradient
counterpart.  Faces are stored per face type (triangle, quad).

The per-point metrics are computed by ``dgb_map_metrics`` on the host cores in threads, one
geometry-basis table per point set (a face group's points are shared by all its faces).  The
inverse mass matrices are not formed here: the operator builds them on the device from w|det J|
(``dgb_plan_build_inverse_mass``); ``ElementPlan.minv`` forms a host copy only when read.
"""

import numpy as np

from . import _native as N
from .mesh import HybridMesh
from .reference import CORNERS, FACE_TYPE_ID, LOCAL_FACES, TYPE_ID, RefElement, face_quadrature, gauss01

FACE_TYPES = ("triangle", "quad")


def _p1_jacobian(etype, xyz, points):
    """J[..., d, r] = sum_k x_k[d] dN_k/dxi_r at reference points (first-order geometry)."""
    g = RefElement(etype, 1).basis_gradients(points)          # (..., 8, 3)
    return np.einsum("...kd,...kr->...dr", xyz, g)


class ElementPlan:
    """Arrays of one element block.  ``minv`` (the dense inverse mass matrices, E * Np^2 values)
    is formed on the host only when read: the device plan builds its own copy from ``wdet``
    (``dgb_plan_build_inverse_mass``)."""

    @property
    def minv(self):
        if getattr(self, "_minv", None) is None:
            m = _inverse_mass(self.wdet, self.ref.B)
            m *= np.minimum(1.0, self.volume / 1.0e-4)[:, None, None]
            self._minv = m
        return self._minv


class FacePlan:
    pass


class Plan:
    """All numpy arrays for one mesh at one polynomial degree."""

    def __init__(self, mesh: HybridMesh, degree: int):
        self.mesh, self.degree = mesh, degree
        self.blocks = [self._element_plan(b, k) for k, b in enumerate(mesh.element_blocks)]
        self.codes = {}          # (etype, ftype) -> list of reference point arrays
        self.faces = {}
        for ftype in FACE_TYPES:
            if ftype in mesh.face_blocks:
                self.faces[ftype] = self._face_plan(ftype, mesh.face_blocks[ftype])
        self._trace_tables()
        self._element_face_links()
        self._lengths()
        self._face_samples()

    # ------------------------------------------------------------ elements
    def _element_plan(self, block, k):
        ref = RefElement(block.element_type, self.degree)
        geo, xyz = self.mesh.geometry(block)                     # (E, n_geometry_nodes, 3)
        # jinv[r][d] = dxi_r/dx_d, wdet = w |det J| at the volume points (host threads)
        det, jinv, wdet = N.map_metrics(xyz, geo.basis_gradients(ref.points), weights=ref.weights,
                                        outputs=("det", "inv_jacobian", "wdet"))
        vol = wdet.sum(axis=1)
        p = ElementPlan()
        p.etype, p.type_id, p.ref = block.element_type, TYPE_ID[block.element_type], ref
        p.E, p.Np, p.Nq = len(block.connectivity), ref.np, ref.nq
        p.nlf = len(LOCAL_FACES[block.element_type])
        p.jinv, p.wdet, p.volume = jinv, wdet, vol
        # one matrix product over all elements: (Np x ng) @ (ng x 3E)
        G = geo.basis(ref.nodes)
        p.node_xyz = np.ascontiguousarray(
            (G @ np.ascontiguousarray(xyz.transpose(1, 0, 2)).reshape(xyz.shape[1], -1))
            .reshape(G.shape[0], xyz.shape[0], 3).transpose(1, 0, 2))
        p.affine = bool(np.all(np.ptp(det, axis=1) <= 1e-13 * np.abs(det).max(axis=1)))
        return p

    # ------------------------------------------------------------ faces
    def _code(self, etype, ftype, pts):
        lst = self.codes.setdefault((etype, ftype), [])
        for c, q in enumerate(lst):
            if q.shape == pts.shape and np.array_equal(q, pts):
                return c
        lst.append(pts)
        return len(lst) - 1

    def _face_plan(self, ftype, fb):
        mesh = self.mesh
        shapes, nweights = face_quadrature(ftype, self.degree)
        F, nq = len(fb.nodes), len(shapes)
        canon = mesh.canon
        fp = FacePlan()
        fp.ftype, fp.F, fp.nq = ftype, F, nq
        fp.owner_block, fp.owner_local = fb.owner_block.copy(), fb.owner_local.copy()
        fp.nbr_block, fp.nbr_local = fb.neighbor_block.copy(), fb.neighbor_local.copy()
        fp.tags = fb.boundary_tags.copy()
        ocode = np.empty(F, np.int32)
        ncode = np.full(F, -1, np.int32)
        normals = np.empty((F, nq, 3))
        weights = np.empty((F, nq))
        jinv_side = np.zeros((F, 2, nq, 3, 3))
        measure = 0.5 if ftype == "triangle" else 1.0
        # Owner side: one point set per (owner type, local face).  The metrics come from the owner
        # mapping (geometry.py:299-353), with the geometry basis evaluated once per point set.
        for b, block in enumerate(mesh.element_blocks):
            geo, xyz_b = mesh.geometry(block)
            for lf, loc in enumerate(LOCAL_FACES[block.element_type]):
                sel = np.flatnonzero((fb.owner_block == b) & (fb.owner_face == lf))
                if not len(sel):
                    continue
                corners = CORNERS[block.element_type][list(loc)]
                pts = shapes @ corners
                ocode[sel] = self._code(block.element_type, ftype, pts)
                if ftype == "triangle":
                    tu = np.broadcast_to(corners[1] - corners[0], pts.shape)
                    tv = np.broadcast_to(corners[2] - corners[0], pts.shape)
                else:
                    u = shapes[:, 1] + shapes[:, 2]
                    v = shapes[:, 2] + shapes[:, 3]
                    c0, c1, c2, c3 = corners
                    tu = -(1 - v)[:, None] * c0 + (1 - v)[:, None] * c1 + v[:, None] * c2 - v[:, None] * c3
                    tv = -(1 - u)[:, None] * c0 - u[:, None] * c1 + u[:, None] * c2 + (1 - u)[:, None] * c3
                # unit normals and w dA from the owner map's tangents J t_u x J t_v, oriented like
                # the face's corner normal (host threads)
                normals[sel], weights[sel], jinv_side[sel, 0] = N.map_metrics(
                    xyz_b, geo.basis_gradients(pts), index=fb.owner_local[sel], weights=nweights * measure,
                    tangents=np.stack([tu, tv], axis=1), orientation=fb.normals[sel],
                    outputs=("normals", "area_weights", "inv_jacobian"))
        # neighbour side: corners matched by canonical node id (geometry.py:205-224)
        internal = np.flatnonzero(fb.neighbor_block >= 0)
        if len(internal):
            k = fb.nodes.shape[1]
            onodes = canon[fb.nodes[internal]]
            nnodes = canon[fb.neighbor_nodes[internal]]
            perm = np.argmax(onodes[:, :, None] == nnodes[:, None, :], axis=2)   # owner corner j -> nbr corner perm[j]
            # (neighbour block, neighbour face, corner permutation) as one integer key: the same
            # order as sorting the tuples
            key = fb.neighbor_block[internal].astype(np.int64) * 8 + fb.neighbor_face[internal]
            for j in range(k):
                key = key * 4 + perm[:, j]
            ukey, inverse = np.unique(key, return_inverse=True)
            uniq = []
            for u in ukey.tolist():
                pm = []
                for _ in range(k):
                    pm.append(u % 4)
                    u //= 4
                uniq.append((u // 8, u % 8, *pm[::-1]))
            for u, (b, lf, *pm) in enumerate(uniq):
                block = mesh.element_blocks[b]
                etype = block.element_type
                corners = CORNERS[etype][list(LOCAL_FACES[etype][lf])][list(pm)]
                pts = shapes @ corners
                faces = internal[inverse == u]
                ncode[faces] = self._code(etype, ftype, pts)
                geo, xyz_b = mesh.geometry(block)
                jinv_side[faces, 1] = N.map_metrics(xyz_b, geo.basis_gradients(pts), index=fb.neighbor_local[faces],
                                                    outputs=("inv_jacobian",))[0]
        fp.ocode, fp.ncode = ocode, ncode
        fp.normals, fp.weights, fp.jinv_side = normals, weights, jinv_side
        return fp

    def _trace_tables(self):
        """Per (element type, face type): basis and reference gradients at each code's points,
        with entries of nodes off the face set to exactly zero."""
        self.trace = {}
        for (etype, ftype), pts_list in self.codes.items():
            ref = RefElement(etype, self.degree)
            B = np.stack([ref.basis(p) for p in pts_list])                  # (C, nq, Np)
            dB = np.stack([ref.basis_gradients(p) for p in pts_list])       # (C, nq, Np, 3)
            for c, p in enumerate(pts_list):
                on_face = _nodes_on_plane(ref.nodes, p)
                B[c][:, ~on_face] = 0.0
            self.trace[(etype, ftype)] = (B, dB)

    def _element_face_links(self):
        """elem_face[e][lf] = (face type << 30) | (face index << 1) | side."""
        for bp in self.blocks:
            bp.elem_face = np.full((bp.E, bp.nlf), -1, np.int64)
        for ftype, fp in self.faces.items():
            ft = FACE_TYPE_ID[ftype]
            fb = self.mesh.face_blocks[ftype]
            f = np.arange(fp.F)
            for side, blk, loc, lf in ((0, fb.owner_block, fb.owner_local, fb.owner_face),
                                       (1, fb.neighbor_block, fb.neighbor_local, fb.neighbor_face)):
                for b, bp in enumerate(self.blocks):
                    sel = np.flatnonzero(blk == b)
                    bp.elem_face[loc[sel], lf[sel]] = (ft << 30) | (f[sel] << 1) | side
        for bp in self.blocks:
            if np.any(bp.elem_face < 0):
                raise ValueError("element face without a face record")
            bp.elem_face = bp.elem_face.astype(np.int32)

    def _lengths(self):
        """time_integration.py:49-91: h = max(2V / sum of face areas, V^(1/3) / (4 (P+1)))."""
        sums = [np.zeros(bp.E) for bp in self.blocks]
        for ftype, fp in self.faces.items():
            area = fp.weights.sum(axis=1)
            for b in range(len(self.blocks)):
                o = np.flatnonzero(fp.owner_block == b)
                np.add.at(sums[b], fp.owner_local[o], area[o])
                n = np.flatnonzero(fp.nbr_block == b)
                np.add.at(sums[b], fp.nbr_local[n], area[n])
        for b, bp in enumerate(self.blocks):
            bp.length = np.maximum(2.0 * bp.volume / sums[b], 0.25 * bp.volume ** (1.0 / 3.0) / (self.degree + 1))

    def _face_samples(self):
        """Distinct face points per element type for the positivity limiter (limiter.py:28-67).

        Every face point of an element type is a point of one of its trace codes, so the
        distinct points are taken over the codes instead of over all faces."""
        for bp in self.blocks:
            chunks = [p for (etype, _), plist in self.codes.items() if etype == bp.etype for p in plist]
            uniq = np.unique(np.round(np.concatenate(chunks), decimals=12), axis=0)
            bp.face_sample_B = bp.ref.basis(uniq)
            p1 = RefElement(bp.etype, 1).basis(bp.ref.nodes)
            bp.p1_projector = p1 @ np.linalg.pinv(p1) if self.degree >= 2 else np.zeros((bp.Np, bp.Np))


def _inverse_mass(wdet, B, chunk=8192):
    """Per-element inverse of M_e = B^T diag(w|J|) B (hybrid/geometry.py:181-188), float64, on the
    host.  The operators build the device copy with ``dgb_plan_build_inverse_mass`` instead."""
    E = wdet.shape[0]
    out = np.empty((E, B.shape[1], B.shape[1]))
    for s in range(0, E, chunk):
        M = np.einsum("eq,qi,qj->eij", wdet[s:s + chunk], B, B, optimize=True)
        out[s:s + chunk] = np.linalg.inv(M)
    return out


def _nodes_on_plane(nodes, pts):
    """Nodes lying on the plane through the face points (all points share one face)."""
    c = pts.mean(axis=0)
    u, s, vt = np.linalg.svd(pts - c)
    normal = vt[-1]
    return np.abs((nodes - c) @ normal) < 1e-9


def _lagrange_1d(nodes, x):
    """1-D Lagrange basis on `nodes` and its derivative at points x: ([len(x)][N], [len(x)][N])."""
    nodes, x = np.asarray(nodes, float), np.atleast_1d(np.asarray(x, float))
    N = len(nodes)
    L = np.ones((len(x), N))
    dL = np.zeros((len(x), N))
    for j in range(N):
        for k in range(N):
            if k == j:
                continue
            f = (x - nodes[k]) / (nodes[j] - nodes[k])
            dL[:, j] = dL[:, j] * f + L[:, j] / (nodes[j] - nodes[k])
            L[:, j] = L[:, j] * f
    return L, dL


def hex_sumfact_tables(plan: Plan):
    """1-D tables, lexicographic node map and face-point permutations of the sum-factorised
    hexahedron path (layout of dgb_plan_set_hex)."""
    P = plan.degree
    bp = plan.blocks[0]
    line = {1: (0.0, 1.0), 2: (0.0, 1.0, 0.5), 3: (0.0, 1.0, 1.0 / 3.0, 2.0 / 3.0)}[P]
    N = P + 1
    Q = len(np.unique(bp.ref.points[:, 0]))
    gq = bp.ref.points[:Q, 0]
    gf, _ = gauss01({1: 2, 2: 3, 3: 4}[P])
    QF = len(gf)
    bq, dq = _lagrange_1d(line, gq)
    bf, df = _lagrange_1d(line, gf)
    _, d01 = _lagrange_1d(line, [0.0, 1.0])

    def pad(a, rows, cols):
        out = np.zeros((rows, cols))
        out[:a.shape[0], :a.shape[1]] = a
        return out.ravel()

    # each block is stored with its real (points x nodes) shape, zero-padded to the capacity
    def packed(a, cap):
        out = np.zeros(cap)
        out[:a.size] = a.ravel()
        return out

    # 1-D mass matrix with the volume Gauss rule (exact: degree 2P <= 2Q - 1) and its inverse; the
    # hexahedron mass matrix of an affine element is det J times its threefold tensor product
    gpts, gw = gauss01(Q)
    assert np.allclose(gpts, gq)
    m1i = np.linalg.inv(np.einsum("q,qi,qj->ij", gw, bq, bq))
    # nodal (Euclidean) projector onto span{1, xi}; on the tensor nodes the sensor's P1 projector
    # (hybrid/limiter.py:158-163, the trilinear functions at the nodes times their pseudo-inverse)
    # is its threefold tensor product
    V1 = np.stack([np.ones(N), np.asarray(line)], axis=1)
    p1d = V1 @ np.linalg.pinv(V1)
    tables = np.concatenate([packed(bq, 20), packed(dq, 20), packed(bq.T.copy(), 20), packed(dq.T.copy(), 20),
                             packed(bf, 16), packed(df, 16), packed(bf.T.copy(), 16),
                             packed(d01[0], 4), packed(d01[1], 4), packed(m1i, 16), packed(gw, 5), packed(p1d, 16)])
    lex = np.full(64, 0, np.int32)
    for iz in range(N):
        for iy in range(N):
            for ix in range(N):
                target = np.array([line[ix], line[iy], line[iz]])
                node = int(np.argmin(np.abs(bp.ref.nodes - target).sum(axis=1)))
                assert np.allclose(bp.ref.nodes[node], target)
                lex[(iz * N + iy) * N + ix] = node
    pts_list = plan.codes.get(("hexahedron", "quad"), [])
    perm = np.zeros((len(pts_list), QF * QF), np.uint8)
    for c, pts in enumerate(pts_list):
        fixed = [a for a in range(3) if np.ptp(pts[:, a]) < 1e-12]
        assert len(fixed) == 1
        a0 = fixed[0]
        a1, a2 = [a for a in range(3) if a != a0]
        k1 = np.argmin(np.abs(pts[:, a1][:, None] - gf[None, :]), axis=1)
        k2 = np.argmin(np.abs(pts[:, a2][:, None] - gf[None, :]), axis=1)
        assert np.max(np.abs(gf[k1] - pts[:, a1])) < 1e-12 and np.max(np.abs(gf[k2] - pts[:, a2])) < 1e-12
        perm[c] = k2 * QF + k1
    return tables, lex, perm, QF * QF


def hex_affine_data(plan: Plan, tol=1.0e-10):
    """Elements of the (single) hexahedron block whose map is affine: the inverse Jacobian is the
    same at every volume point to ``tol`` relative.  Returns (affine uint8[E], coef[E] = sliver
    scale / det J, jinv[E][9], det[E]) in the layout of dgb_plan_set_hex_affine; for those
    elements the inverse mass matrix is coef * (m1i (x) m1i (x) m1i)."""
    cached = plan.__dict__.get("_hex_affine")
    if cached is not None and cached[0] == tol:
        return cached[1]
    bp = plan.blocks[0]
    J = bp.jinv.reshape(bp.E, bp.Nq, 9)
    affine, mean = _affine_test(J, tol)
    det = bp.volume.astype(np.float64)              # the reference hexahedron [0, 1]^3 has volume 1
    coef = np.minimum(1.0, bp.volume / 1.0e-4) / det
    out = affine, coef, mean, det
    plan._hex_affine = (tol, out)                   # shared by the plans of both precisions
    return out


def _affine_test(J, tol):
    """Per element of J (E, Nq, 9): whether every point's inverse Jacobian equals the first one's to
    ``tol`` relative to the largest entry, and the mean over the points (host threads)."""
    return N.affine_test(J, tol)


def block_affine_data(bp, tol=1.0e-10):
    """Elements of one block whose map is affine (the inverse Jacobian is the same at every volume
    point to ``tol`` relative) for the dense path: (affine uint8[E], coef[E] = sliver scale /
    |det J|, jinv[E][9], |det J|[E], reference weights [Nq], inverse reference mass [Np][Np]) in
    the layout of dgb_plan_set_block_affine.  For those elements w_q |det J| = w_q * det and the
    inverse mass matrix (hybrid/geometry.py:181-192) is coef * inv(B^T diag(w) B)."""
    J = bp.jinv.reshape(bp.E, bp.Nq, 9)
    affine, mean = _affine_test(J, tol)
    w = np.asarray(bp.ref.weights, np.float64)
    det = bp.volume / w.sum()
    coef = np.minimum(1.0, bp.volume / 1.0e-4) / det
    mref = np.einsum("q,qi,qj->ij", w, bp.ref.B, bp.ref.B)
    return affine, coef, mean, det, w, np.linalg.inv(mref)
