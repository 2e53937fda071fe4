"""Host plan of the MOOD subcell finite-volume fallback.

Follows ``hybrid/subcell.py`` of superboss2300/jax-fluid-sim: every element is
split into 64 reference subcells (4 divisions per edge: hexahedra into 4^3
cubes, wedges into 16 triangles x 4 layers, tetrahedra by two red
refinements); per element the metric-weighted projection DG -> subcell means
(P2 volume rule mapped onto each subcell), its volume-weighted least-squares
left inverse, subcell volumes, centres and face metrics; per parent face the
16 boundary subfaces of each side, the neighbour's matched to the owner's by
physical centre.

Coupling indices: the reference reads and writes subcell arrays with the
boundary-subface ids of a parent face (``subcell.py:774-775,803-805,836-843``);
under JAX an id past the last subcell is clamped when read and dropped when
written.  ``coupling="reference"`` reproduces that; ``coupling="subcell"``
uses the subcell owning each subface.
"""

import ctypes
import os
import threading

import numpy as np

from . import _native as N
from .reference import LOCAL_FACES, RefElement, volume_quadrature

DIVISIONS = 4


def _hex_cells(n):
    verts = np.array([(i, j, k) for k in range(n + 1) for j in range(n + 1) for i in range(n + 1)], float) / n
    idx = lambda i, j, k: (k * (n + 1) + j) * (n + 1) + i
    cells = [[idx(i, j, k), idx(i + 1, j, k), idx(i + 1, j + 1, k), idx(i, j + 1, k),
              idx(i, j, k + 1), idx(i + 1, j, k + 1), idx(i + 1, j + 1, k + 1), idx(i, j + 1, k + 1)]
             for k in range(n) for j in range(n) for i in range(n)]
    return verts, np.array(cells, np.int32)


def _wedge_cells(n):
    tri = [(i / n, j / n) for i in range(n + 1) for j in range(n + 1 - i)]
    where = {(round(x * n), round(y * n)): k for k, (x, y) in enumerate(tri)}
    tris = []
    for i in range(n):
        for j in range(n - i):
            tris.append((where[i, j], where[i + 1, j], where[i, j + 1]))
            if i + j <= n - 2:
                tris.append((where[i + 1, j], where[i + 1, j + 1], where[i, j + 1]))
    verts = np.array([(x, y, l / n) for l in range(n + 1) for x, y in tri], float)
    m = len(tri)
    cells = [[l * m + a, l * m + b, l * m + c, (l + 1) * m + a, (l + 1) * m + b, (l + 1) * m + c]
             for l in range(n) for a, b, c in tris]
    return verts, np.array(cells, np.int32)


def _tet_cells():
    verts = [(0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)]
    index = {v: k for k, v in enumerate(verts)}
    cells = [(0, 1, 2, 3)]
    for _ in range(2):
        def mid(a, b):
            p = tuple(0.5 * (np.array(verts[a]) + np.array(verts[b])))
            if p not in index:
                index[p] = len(verts)
                verts.append(p)
            return index[p]
        new = []
        for a, b, c, d in cells:
            ab, ac, ad, bc, bd, cd = mid(a, b), mid(a, c), mid(a, d), mid(b, c), mid(b, d), mid(c, d)
            new += [(a, ab, ac, ad), (ab, b, bc, bd), (ac, bc, c, cd), (ad, bd, cd, d),
                    (ab, ac, ad, bd), (ab, bc, ac, bd), (ac, ad, bd, cd), (ac, bd, bc, cd)]
        cells = new
    return np.array(verts, float), np.array(cells, np.int32)


def _on_parent_face(etype, pts):
    x, y, z = pts[:, 0], pts[:, 1], pts[:, 2]
    tests = {"tetra": (z, y, x + y + z - 1.0, x), "wedge": (z, z - 1.0, y, x + y - 1.0, x),
             "hexahedron": (z, z - 1.0, y, x - 1.0, y - 1.0, x)}[etype]
    for f, t in enumerate(tests):
        if np.all(np.abs(t) <= 1e-10):
            return f
    return -1


class ReferenceSubcells:
    """Subcell vertices/cells, internal subfaces (owner, neighbour, vertex list) in the order
    the reference pairs them, boundary subfaces with their parent face."""

    def __init__(self, etype):
        self.etype = etype
        if etype == "hexahedron":
            self.vertices, self.cells = _hex_cells(DIVISIONS)
        elif etype == "wedge":
            self.vertices, self.cells = _wedge_cells(DIVISIONS)
        else:
            self.vertices, self.cells = _tet_cells()
        pending, own, nbr, ifaces = {}, [], [], []
        for c, conn in enumerate(self.cells):
            for loc in LOCAL_FACES[etype]:
                face = conn[list(loc)]
                key = tuple(sorted(face.tolist()))
                if key in pending:
                    oc, of = pending.pop(key)
                    own.append(oc)
                    nbr.append(c)
                    ifaces.append(of)
                else:
                    pending[key] = (c, face)
        self.internal_owner = np.array(own, np.int32)
        self.internal_neighbor = np.array(nbr, np.int32)
        self.internal_faces = ifaces
        self.boundary_owner = np.array([c for c, _ in pending.values()], np.int32)
        self.boundary_faces = [f for _, f in pending.values()]
        self.boundary_parent = np.array([_on_parent_face(etype, self.vertices[f]) for f in self.boundary_faces],
                                        np.int32)
        if np.any(self.boundary_parent < 0):
            raise ValueError("Subcell boundary face is not on its parent boundary")
        self.count = len(self.cells)
        self.boundary_reference_centers = np.array([self.vertices[f].mean(axis=0) for f in self.boundary_faces])
        # CSR of internal subfaces per subcell (for gather-based sums)
        inc = [[] for _ in range(self.count)]
        for k, (a, b) in enumerate(zip(own, nbr)):
            inc[a].append(k)
            inc[b].append(k)
        self.csr_ptr = np.cumsum([0] + [len(x) for x in inc]).astype(np.int32)
        self.csr_face = np.array([k for x in inc for k in x], np.int32)

    def coupling_indices(self, mode):
        """Per boundary subface: subcell read (gather) and subcell written (scatter, -1 = none)."""
        k = np.arange(len(self.boundary_faces))
        if mode == "subcell":
            return self.boundary_owner.copy(), self.boundary_owner.copy()
        if mode != "reference":
            raise ValueError("coupling must be 'reference' or 'subcell'")
        return np.minimum(k, self.count - 1).astype(np.int32), np.where(k < self.count, k, -1).astype(np.int32)


def _subcell_rule(rs):
    """P2 volume rule mapped affinely onto each reference subcell (subcell.py:236-274)."""
    pts, wts = volume_quadrature(rs.etype, 2)
    cv = rs.vertices[rs.cells]
    mapped = np.einsum("qi,sir->sqr", RefElement(rs.etype, 1).basis(pts), cv)
    cols = (1, 3, 4) if rs.etype == "hexahedron" else (1, 2, 3)
    mats = np.stack([cv[:, c] - cv[:, 0] for c in cols], axis=-1)
    return mapped, wts[None, :] * np.abs(np.linalg.det(mats))[:, None]


class SubcellBlockPlan:
    """Per-element subcell geometry of one block (float64)."""

    def __init__(self, mesh, block, degree, rs, chunk=4096):
        etype = block.element_type
        ref = RefElement(etype, degree)
        geo1, xyz_all = mesh.geometry(block)          # subcell.py:282-288: the block's geometry map
        mp, rw = _subcell_rule(rs)
        flat = mp.reshape(-1, 3)
        sb = ref.basis(flat).reshape(rs.count, mp.shape[1], -1)
        vb = geo1.basis(rs.vertices)
        E = len(block.connectivity)
        S, Np = rs.count, ref.np
        self.projection = np.empty((E, S, Np))
        self.reconstruction = np.empty((E, Np, S))
        self.volumes = np.empty((E, S))
        self.centers = np.empty((E, S, 3))
        NI, NB = len(rs.internal_faces), len(rs.boundary_faces)
        self.internal_normals = np.empty((E, NI, 3))
        self.internal_areas = np.empty((E, NI))
        self.boundary_normals = np.empty((E, NB, 3))
        self.boundary_areas = np.empty((E, NB))
        self.boundary_centers = np.empty((E, NB, 3))
        gflat = geo1.basis_gradients(flat)                 # (S * Qs, n, 3)
        Qs = mp.shape[1]
        import torch
        device = torch.cuda.current_device() if torch.cuda.is_available() else None

        # Chunks of elements are independent and write disjoint rows, so they run in host threads
        # (numpy and the native routines release the interpreter lock); each chunk's arithmetic is
        # the same whichever thread takes it.
        def work(s0):
            xyz = xyz_all[s0:s0 + chunk]
            e = len(xyz)
            pv = np.einsum("vi,eid->evd", vb, xyz)
            cen = pv[:, rs.cells].mean(axis=2)
            # subcell.py:308-323: |det J| at the mapped subcell points (host threads), subcell
            # volumes and the metric-weighted projection; matrix products per subcell / element
            det = N.map_metrics(xyz, gflat, outputs=("det",))[0]
            pw = np.abs(det).reshape(e, S, Qs) * rw[None]
            vol = pw.sum(axis=-1)
            # (contiguous operands, so that each product of the stack goes to BLAS)
            proj = np.matmul(np.ascontiguousarray(pw.transpose(1, 0, 2)), sb).transpose(1, 0, 2) / vol[..., None]
            # subcell.py:324-334: volume-weighted least-squares left inverse
            wpT = np.ascontiguousarray((proj * vol[..., None]).transpose(0, 2, 1))     # (e, Np, S)
            gram = np.matmul(wpT, proj)
            rec = np.matmul(_spd_inverse(gram, device), wpT)
            sl = slice(s0, s0 + e)
            self.projection[sl], self.reconstruction[sl], self.volumes[sl], self.centers[sl] = proj, rec, vol, cen
            n, a, _ = _face_metrics(pv, cen, rs.internal_faces, rs.internal_owner, rs.internal_neighbor)
            self.internal_normals[sl], self.internal_areas[sl] = n, a
            n, a, c = _face_metrics(pv, cen, rs.boundary_faces, rs.boundary_owner, None)
            self.boundary_normals[sl], self.boundary_areas[sl], self.boundary_centers[sl] = n, a, c

        starts = range(0, E, chunk)
        if len(starts) > 1:
            from concurrent.futures import ThreadPoolExecutor
            with ThreadPoolExecutor(max_workers=min(len(starts), os.cpu_count() or 1, 8)) as pool:
                list(pool.map(work, starts))
        else:
            for s0 in starts:
                work(s0)
        self.boundary_basis = ref.basis(rs.boundary_reference_centers)    # [NB][Np]


_GPU_LOCK = threading.Lock()


def _spd_inverse(gram, device):
    """Inverses of a stack of SPD matrices: on GPU ``device`` (``dgb_spd_inverse``) when one is
    given, else with numpy (set-up only).  The choice does not depend on the stack's size, so an
    element gets the same matrix whichever mesh or chunk it is part of.  Host threads take the GPU
    one at a time, each first making ``device`` its current device (that setting is per thread)."""
    if device is None or len(gram) == 0:
        return np.linalg.inv(gram)
    import torch
    with _GPU_LOCK:
        torch.cuda.set_device(device)
        return _spd_inverse_gpu(torch, gram)


def _spd_inverse_gpu(torch, gram):
    t = torch.as_tensor(np.ascontiguousarray(gram), device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    N.check(N.lib().dgb_spd_inverse(ctypes.c_void_p(t.data_ptr()), gram.shape[1], len(gram),
                                    ctypes.c_void_p(status.data_ptr()),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    if int(status.item()):
        raise ValueError(f"subcell Gram matrix {int(status.item()) - 1} of the chunk is not positive definite")
    return t.cpu().numpy()


def _face_metrics(pv, cen, faces, owners, neighbors):
    """Unit normals, areas and centres of subcell faces, area vectors oriented owner -> neighbour
    (or outward) (subcell.py:336-360), on the host cores (``dgb_subcell_face_metrics``)."""
    return N.subcell_face_metrics(pv, cen, faces, owners, neighbors)


def _padded_faces(faces):
    out = np.full((len(faces), 4), -1, np.int32)
    for k, f in enumerate(faces):
        out[k, :len(f)] = f
    return out


def device_reference(mesh, block, degree, rs):
    """Reference tables from which the device builds a block's subcell tables
    (``dgb_plan_build_subcells``): the subcells' P2 rule (weights times each subcell's reference
    volume factor), the DG basis and the geometry-basis gradients at the mapped points, the
    geometry basis at the subcell vertices, the subcell vertex lists and the padded subface
    vertex lists; plus the block's geometry-map nodes (E, ng, 3)."""
    ref = RefElement(block.element_type, degree)
    geo1, xyz_all = mesh.geometry(block)
    mp, rw = _subcell_rule(rs)
    flat = mp.reshape(-1, 3)
    S, Qs = mp.shape[0], mp.shape[1]
    tables = dict(rule_weights=rw, point_basis=ref.basis(flat).reshape(S, Qs, ref.np),
                  point_geometry_grad=geo1.basis_gradients(flat), vertex_geometry=geo1.basis(rs.vertices),
                  cells=rs.cells, internal_faces=_padded_faces(rs.internal_faces),
                  boundary_faces=_padded_faces(rs.boundary_faces), boundary_basis=ref.basis(rs.boundary_reference_centers))
    return tables, np.ascontiguousarray(xyz_all, np.float64)


def subface_tables(mesh, refs):
    """Per face type: the owner's 16 boundary subfaces on the parent face (osub) and the
    neighbour's 16 on its side of it in reference order (ncand, -1 on boundary faces), which the
    device matches to the owner's by centre (``dgb_plan_match_subcell_faces``)."""
    out = {}
    for ftype, fb in mesh.face_blocks.items():
        F = len(fb.nodes)
        osub = np.zeros((F, 16), np.int32)
        ncand = np.full((F, 16), -1, np.int32)
        for b, block in enumerate(mesh.element_blocks):
            rs = refs[block.element_type]
            for lf in range(len(LOCAL_FACES[block.element_type])):
                ids = np.flatnonzero(rs.boundary_parent == lf).astype(np.int32)
                if len(ids) != 16:
                    continue
                osub[(fb.owner_block == b) & (fb.owner_face == lf)] = ids
                ncand[(fb.neighbor_block == b) & (fb.neighbor_face == lf)] = ids
        out[ftype] = (osub, ncand)
    return out


class SubcellPlan:
    """Subcell tables of a whole mesh plus the per-face subface lists of both sides, built on the
    host (numpy, the native metrics and the GPU Gram inverses): the construction the device build
    is tested against."""

    def __init__(self, mesh, degree, coupling="reference"):
        self.coupling = coupling
        self.refs = {b.element_type: ReferenceSubcells(b.element_type) for b in mesh.element_blocks}
        self.blocks = [SubcellBlockPlan(mesh, b, degree, self.refs[b.element_type]) for b in mesh.element_blocks]
        self.faces = {}
        for ftype, fb in mesh.face_blocks.items():
            F = len(fb.nodes)
            osub = np.zeros((F, 16), np.int32)
            nsub = np.full((F, 16), -1, np.int32)
            for b, block in enumerate(mesh.element_blocks):
                rs = self.refs[block.element_type]
                for lf in range(len(LOCAL_FACES[block.element_type])):
                    ids = np.flatnonzero(rs.boundary_parent == lf).astype(np.int32)
                    sel = np.flatnonzero((fb.owner_block == b) & (fb.owner_face == lf))
                    if len(sel) and len(ids) == 16:
                        osub[sel] = ids
            # neighbour subfaces matched to the owner's by physical centre; centres are taken
            # relative to each side's face centre so periodic partners match as well
            for b in range(len(mesh.element_blocks)):
                for nf in range(len(LOCAL_FACES[mesh.element_blocks[b].element_type])):
                    sel = np.flatnonzero((fb.neighbor_block == b) & (fb.neighbor_face == nf))
                    if not len(sel):
                        continue
                    rsn = self.refs[mesh.element_blocks[b].element_type]
                    nids = np.flatnonzero(rsn.boundary_parent == nf).astype(np.int32)
                    oxyz = np.stack([self.blocks[ob].boundary_centers[ol, osub[f]] for f, ob, ol in
                                     zip(sel, fb.owner_block[sel], fb.owner_local[sel])]) if len(mesh.element_blocks) > 1 \
                        else self.blocks[0].boundary_centers[fb.owner_local[sel][:, None], osub[sel]]
                    nxyz = self.blocks[b].boundary_centers[fb.neighbor_local[sel][:, None], nids[None, :]]
                    oc, nc = oxyz.mean(axis=1, keepdims=True), nxyz.mean(axis=1, keepdims=True)
                    d = np.linalg.norm((oxyz - oc)[:, :, None, :] - (nxyz - nc)[:, None, :, :], axis=-1)
                    perm = np.argmin(d, axis=2)
                    best = np.take_along_axis(d, perm[..., None], axis=2)[..., 0]
                    scale = np.maximum(np.max(np.linalg.norm(oxyz, axis=2), axis=1), 1.0)
                    distinct = np.all(np.sort(perm, axis=1) == np.arange(16)[None, :], axis=1)
                    if not np.all(distinct) or np.any(best.max(axis=1) > 2e-6 * scale):
                        raise ValueError(f"Nonconforming subfaces at {ftype} faces")
                    nsub[sel] = nids[perm]
            self.faces[ftype] = (osub, nsub)
