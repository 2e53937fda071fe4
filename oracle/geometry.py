"""Isoparametric element and face metrics (first-order geometry).

Oracle restatement of ``hybrid/geometry.py``:
* element metrics: mapped points, J = x (x) grad N, det, inv, w|J|, physical
  basis gradients, mass, sliver-scaled inverse mass (``:139-203``);
* solution-node coordinates (``:115-137``);
* face metrics: owner reference points from the owner's local-face corners,
  neighbour points from corners matched by (canonical) node id, tangents
  mapped by the owner Jacobian, area vector oriented like the mesh normal,
  weights = normalised rule x reference measure x |area vector|
  (``:205-362``).
Blocks of complete second-order cells use the second-order reference element as
the geometry basis on their geometry nodes (``:102-110``); all others the first-order one.
"""

import numpy as np

from .elements import RefElement, corner_nodes, face_quadrature
from .mesh import LOCAL_FACES


class ElementMetrics:
    pass


class FaceMetrics:
    pass


class Geometry:
    def __init__(self, mesh, degree):
        self.mesh = mesh
        self.degree = degree
        types = {b.element_type for b in mesh.element_blocks}
        self.ref = {t: RefElement(t, degree) for t in types}
        self.geo_ref = {b.element_type: RefElement(b.element_type, 1 if b.geometry_connectivity is None else 2)
                        for b in mesh.element_blocks}
        self.element = [self._element_metrics(b) for b in mesh.element_blocks]
        self.node_xyz = {}
        for b in mesh.element_blocks:
            gb = self.geo_ref[b.element_type].basis(self.ref[b.element_type].nodes)
            self.node_xyz[b.element_type] = np.einsum("qi,eid->eqd", gb, self.geometry_nodes(b))
        self.face = {ft: self._face_metrics(ft, fb) for ft, fb in mesh.face_blocks.items()}

    def geometry_nodes(self, block):
        return self.mesh.points[block.connectivity if block.geometry_connectivity is None
                                else block.geometry_connectivity]

    def _element_metrics(self, block):
        ref, gref = self.ref[block.element_type], self.geo_ref[block.element_type]
        xyz = self.geometry_nodes(block)
        gb = gref.basis(ref.volume_points)
        gg = gref.basis_gradients(ref.volume_points)
        m = ElementMetrics()
        m.points = np.einsum("qi,eid->eqd", gb, xyz)
        m.jacobian = np.einsum("eid,qir->eqdr", xyz, gg)
        m.det = np.linalg.det(m.jacobian)
        m.inv = np.linalg.inv(m.jacobian)
        m.grad = np.einsum("qir,eqrd->eqid", ref.dB, m.inv)
        m.wdet = ref.volume_weights[None, :] * np.abs(m.det)
        m.mass = np.einsum("eq,qi,qj->eij", m.wdet, ref.B, ref.B)
        minv = np.linalg.inv(m.mass)
        vols = m.wdet.sum(axis=1)
        m.minv = np.minimum(1.0, vols / 1.0e-4)[:, None, None] * minv
        m.volumes = vols
        return m

    def aligned_neighbor_corners(self, fb, f, owner_nodes):
        nb = int(fb.neighbor_block[f])
        if nb < 0:
            return np.full((len(owner_nodes), 3), np.nan)
        block = self.mesh.element_blocks[nb]
        loc = LOCAL_FACES[block.element_type][int(fb.neighbor_face[f])]
        nnodes = block.connectivity[int(fb.neighbor_local[f]), list(loc)]
        nref = corner_nodes(block.element_type)[list(loc)]
        canon = self.mesh.canon
        lookup = {int(canon[n]): nref[k] for k, n in enumerate(nnodes)}
        return np.asarray([lookup[int(canon[n])] for n in owner_nodes])

    def _face_metrics(self, ftype, fb):
        shapes, nweights = face_quadrature(ftype, self.degree)
        own_pts, nbr_pts, tu_ref, tv_ref = [], [], [], []
        for f, onodes in enumerate(fb.nodes):
            oblock = self.mesh.element_blocks[int(fb.owner_block[f])]
            corners = corner_nodes(oblock.element_type)[list(LOCAL_FACES[oblock.element_type][int(fb.owner_face[f])])]
            own_pts.append(shapes @ corners)
            nbr_pts.append(shapes @ self.aligned_neighbor_corners(fb, f, onodes))
            p = shapes @ corners
            if ftype == "triangle":
                tu = np.broadcast_to(corners[1] - corners[0], p.shape)
                tv = np.broadcast_to(corners[2] - corners[0], p.shape)
            else:
                u = shapes[:, 1] + shapes[:, 2]
                v = shapes[:, 2] + shapes[:, 3]
                c0, c1, c2, c3 = corners
                tu = -(1 - v)[:, None] * c0 + (1 - v)[:, None] * c1 + v[:, None] * c2 - v[:, None] * c3
                tv = -(1 - u)[:, None] * c0 - u[:, None] * c1 + u[:, None] * c2 + (1 - u)[:, None] * c3
            tu_ref.append(tu)
            tv_ref.append(tv)
        own_pts, nbr_pts = np.asarray(own_pts), np.asarray(nbr_pts)
        tu_ref, tv_ref = np.asarray(tu_ref), np.asarray(tv_ref)
        nf, nq = own_pts.shape[:2]
        pts = np.zeros((nf, nq, 3))
        normals = np.zeros((nf, nq, 3))
        weights = np.zeros((nf, nq))
        measure = 0.5 if ftype == "triangle" else 1.0
        for ob in np.unique(fb.owner_block):
            idx = np.flatnonzero(fb.owner_block == ob)
            block = self.mesh.element_blocks[int(ob)]
            gref = self.geo_ref[block.element_type]
            xyz = self.geometry_nodes(block)[fb.owner_local[idx]]
            gb = gref.basis(own_pts[idx])
            gg = gref.basis_gradients(own_pts[idx])
            mapped = np.einsum("fqi,fid->fqd", gb, xyz)
            jac = np.einsum("fid,fqir->fqdr", xyz, gg)
            tu = np.einsum("fqdr,fqr->fqd", jac, tu_ref[idx])
            tv = np.einsum("fqdr,fqr->fqd", jac, tv_ref[idx])
            area = np.cross(tu, tv)
            sign = np.where(np.sum(area * fb.normals[idx][:, None, :], axis=-1) >= 0, 1.0, -1.0)
            area = area * sign[..., None]
            mag = np.linalg.norm(area, axis=-1)
            pts[idx] = mapped
            normals[idx] = area / mag[..., None]
            weights[idx] = nweights[None, :] * measure * mag
        m = FaceMetrics()
        m.points, m.normals, m.weights = pts, normals, weights
        m.owner_points, m.neighbor_points = own_pts, nbr_pts
        return m

    def physical_basis_gradients(self, block_id, cells, points):
        """navier_stokes.py:112-136: grad phi at arbitrary reference points, J inverted per point."""
        block = self.mesh.element_blocks[block_id]
        ref, gref = self.ref[block.element_type], self.geo_ref[block.element_type]
        xyz = self.geometry_nodes(block)[cells]
        jac = np.einsum("fid,fqir->fqdr", xyz, gref.basis_gradients(points))
        return np.einsum("fqir,fqrd->fqid", ref.basis_gradients(points), np.linalg.inv(jac))
