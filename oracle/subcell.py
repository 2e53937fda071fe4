"""MOOD subcell finite-volume recompute on the CPU (oracle).

Restatement of ``hybrid/subcell.py`` and ``hybrid/limiter.py:267-343``:
* reference subcells: 4 divisions per edge, hexahedra 4^3 cubes, wedges 16
  triangles x 4 layers, tetrahedra two red refinements (``subcell.py:53-233``);
* metric-weighted projection DG -> subcell means and its volume-weighted
  least-squares left inverse (``:236-396``), subcell face metrics;
* bound-limited reconstruction back to DG (``:406-439``);
* internal fluxes with constant / TVD / CWENO-Z reconstruction and
  admissibility clamps (``:541-688``);
* DG-FV coupling fluxes on parent faces, the original DG face flux and the
  conservative correction of untroubled neighbours (``:473-533,690-950``);
* MOOD limiter: troubled detection on the unlimited candidate, recompute,
  positivity (``limiter.py:267-343``) and the MOOD branch of checked_step
  (``time_integration.py:450-554``).
"""

import numpy as np

from .dg import PositivityLimiter, TroubledCellSensor, mood_troubled
from .elements import basis as _basis, basis_gradients as _basis_grad, volume_quadrature
from .mesh import LOCAL_FACES


# ------------------------------------------------------------------ reference subcells
def _triangle_lattice(n):
    verts = np.asarray([(i / n, j / n) for i in range(n + 1) for j in range(n + 1 - i)], float)
    lookup = {tuple(np.rint(p * n).astype(int)): k for k, p in enumerate(verts)}
    tris = []
    for i in range(n):
        for j in range(n - i):
            tris.append([lookup[(i, j)], lookup[(i + 1, j)], lookup[(i, j + 1)]])
            if i + j <= n - 2:
                tris.append([lookup[(i + 1, j)], lookup[(i + 1, j + 1)], lookup[(i, j + 1)]])
    return verts, np.asarray(tris, np.int32)


def _tetra_subdivision():
    verts = [np.array(v, float) for v in ([0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1])]
    cells = [(0, 1, 2, 3)]
    for _ in range(2):
        lookup = {tuple(p): i for i, p in enumerate(verts)}

        def mid(a, b):
            p = 0.5 * (verts[a] + verts[b])
            k = tuple(p)
            if k not in lookup:
                lookup[k] = len(verts)
                verts.append(p)
            return lookup[k]

        out = []
        for a, b, c, d in cells:
            ab, ac, ad, bc, bd, cd = mid(a, b), mid(a, c), mid(a, d), mid(b, c), mid(b, d), mid(c, d)
            out += [(a, ab, ac, ad), (ab, b, bc, bd), (ac, bc, c, cd), (ad, bd, cd, d),
                    (ab, ac, ad, bd), (ab, bc, ac, bd), (ac, ad, bd, cd), (ac, bd, bc, cd)]
        cells = out
    return np.asarray(verts), np.asarray(cells, np.int32)


def _wedge_subdivision(n):
    tv, tris = _triangle_lattice(n)
    verts = np.asarray([(x, y, layer / n) for layer in range(n + 1) for x, y in tv], float)
    ls = len(tv)
    cells = [[lo + a, lo + b, lo + c, lo + ls + a, lo + ls + b, lo + ls + c]
             for lo in (layer * ls for layer in range(n)) for a, b, c in tris]
    return verts, np.asarray(cells, np.int32)


def _hex_subdivision(n):
    verts = np.asarray([(i / n, j / n, k / n) for k in range(n + 1) for j in range(n + 1) for i in range(n + 1)], float)

    def idx(i, j, k):
        return k * (n + 1) ** 2 + j * (n + 1) + i

    cells = [[idx(i, j, k), idx(i + 1, j, k), idx(i + 1, j + 1, k), idx(i, j + 1, k),
              idx(i, j, k + 1), idx(i + 1, j, k + 1), idx(i + 1, j + 1, k + 1), idx(i, j + 1, k + 1)]
             for k in range(n) for j in range(n) for i in range(n)]
    return verts, np.asarray(cells, np.int32)


def _parent_face(etype, xyz, tol=1e-10):
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    tests = {"tetra": (z, y, x + y + z - 1.0, x), "wedge": (z, z - 1.0, y, x + y - 1.0, x),
             "hexahedron": (z, z - 1.0, y, x - 1.0, y - 1.0, x)}[etype]
    for f, v in enumerate(tests):
        if np.all(np.abs(v) <= tol):
            return f
    return -1


class RefSubcells:
    """subcell.py:20-233 (division count 4)."""

    def __init__(self, etype, n=4):
        if etype == "tetra":
            self.vertices, self.cells = _tetra_subdivision()
        elif etype == "wedge":
            self.vertices, self.cells = _wedge_subdivision(n)
        else:
            self.vertices, self.cells = _hex_subdivision(n)
        self.etype = etype
        pending = {}
        io, ineigh, ifaces, bo, bparent, bfaces = [], [], [], [], [], []
        for c, conn in enumerate(self.cells):
            for loc in LOCAL_FACES[etype]:
                face = np.asarray(conn[list(loc)], np.int32)
                key = tuple(sorted(int(v) for v in face))
                if key in pending:
                    oc, of = pending.pop(key)
                    io.append(oc)
                    ineigh.append(c)
                    ifaces.append(of)
                else:
                    pending[key] = (c, face)
        for c, face in pending.values():
            pf = _parent_face(etype, self.vertices[face])
            if pf < 0:
                raise ValueError("Subcell boundary face is not on its parent boundary")
            bo.append(c)
            bparent.append(pf)
            bfaces.append(face)
        self.internal_owner, self.internal_neighbor = np.asarray(io, np.int32), np.asarray(ineigh, np.int32)
        self.internal_faces, self.boundary_faces = tuple(ifaces), tuple(bfaces)
        self.boundary_owner, self.boundary_parent = np.asarray(bo, np.int32), np.asarray(bparent, np.int32)
        self.count = len(self.cells)


def _mapped_quadrature(rs):
    """subcell.py:236-274: P2 volume rule mapped affinely onto each reference subcell."""
    pts, wts = volume_quadrature(rs.etype, 2)
    cv = rs.vertices[rs.cells]
    mapped = np.einsum("qi,sir->sqr", _basis(rs.etype, 1, pts), cv)
    if rs.etype == "hexahedron":
        mats = np.stack([cv[:, 1] - cv[:, 0], cv[:, 3] - cv[:, 0], cv[:, 4] - cv[:, 0]], axis=-1)
    else:
        mats = np.stack([cv[:, 1] - cv[:, 0], cv[:, 2] - cv[:, 0], cv[:, 3] - cv[:, 0]], axis=-1)
    return mapped, wts[None, :] * np.abs(np.linalg.det(mats))[:, None]


class SubcellProjection:
    """subcell.py:277-396 for one element block."""

    def __init__(self, op, block_id, rs):
        mesh, geo = op.mesh, op.geo
        block = mesh.element_blocks[block_id]
        etype = block.element_type
        gdeg = 1 if block.geometry_connectivity is None else 2          # subcell.py:282-288
        xyz = geo.geometry_nodes(block)
        pv = np.einsum("vi,eid->evd", _basis(etype, gdeg, rs.vertices), xyz)
        cells_xyz = pv[:, rs.cells]
        self.centers = cells_xyz.mean(axis=2)
        mp, rw = _mapped_quadrature(rs)
        flat = mp.reshape(-1, 3)
        sb = _basis(etype, op.degree, flat).reshape(rs.count, mp.shape[1], -1)
        gg = _basis_grad(etype, gdeg, flat).reshape(rs.count, mp.shape[1], -1, 3)
        jac = np.einsum("eir,sqij->esqrj", xyz, gg)
        pw = np.abs(np.linalg.det(jac)) * rw[None]
        self.volumes = pw.sum(axis=-1)
        self.projection = np.einsum("esq,sqi->esi", pw, sb) / self.volumes[..., None]
        gram = np.einsum("esi,es,esj->eij", self.projection, self.volumes, self.projection)
        self.reconstruction = np.einsum("eij,esj,es->eis", np.linalg.inv(gram), self.projection, self.volumes)

        def face_metrics(faces, owners, neighbors=None):
            av, cen = [], []
            for face in faces:
                p = pv[:, np.asarray(face)]
                c = p.mean(axis=1)
                a = 0.5 * np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
                if len(face) == 4:
                    a = a + 0.5 * np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0])
                av.append(a)
                cen.append(c)
            av, cen = np.stack(av, axis=1), np.stack(cen, axis=1)
            oc = self.centers[:, owners]
            direction = cen - oc if neighbors is None else self.centers[:, neighbors] - oc
            av = av * np.where(np.sum(av * direction, axis=-1) >= 0.0, 1.0, -1.0)[..., None]
            ar = np.linalg.norm(av, axis=-1)
            return av / ar[..., None], ar, cen

        self.internal_normals, self.internal_areas, _ = face_metrics(rs.internal_faces, rs.internal_owner,
                                                                     rs.internal_neighbor)
        self.boundary_normals, self.boundary_areas, self.boundary_centers = face_metrics(rs.boundary_faces,
                                                                                         rs.boundary_owner)
        self.boundary_reference_centers = np.asarray([rs.vertices[f].mean(axis=0) for f in rs.boundary_faces])


def subcells_to_dg(avg, proj, bound_limit=True):
    """subcell.py:406-439."""
    raw = np.einsum("eis,esv->eiv", proj.reconstruction, avg)
    if not bound_limit:
        return raw
    vols = proj.volumes
    mean = np.sum(avg * vols[..., None], axis=1) / np.maximum(vols.sum(axis=1, keepdims=True), 1e-14)
    smin, smax = avg.min(axis=1), avg.max(axis=1)
    dmin, dmax = raw.min(axis=1), raw.max(axis=1)
    eps = 1e-12
    with np.errstate(all="ignore"):
        tmax = np.where(dmax > mean + eps, (smax - mean) / (dmax - mean + eps), 1.0)
        tmin = np.where(dmin < mean - eps, (mean - smin) / (mean - dmin + eps), 1.0)
    theta = np.clip(np.minimum(tmax, tmin), 0.0, 1.0)
    return mean[:, None, :] + theta[:, None, :] * (raw - mean[:, None, :])


def _clamp(U):
    """Admissibility clamps on reconstructed traces (subcell.py:645-663)."""
    U = U.copy()
    U[..., 0] = np.maximum(U[..., 0], 1e-14)
    ek = 0.5 * np.sum(U[..., 1:4] ** 2, axis=-1) / U[..., 0]
    U[..., 4] = np.maximum(U[..., 4], ek + 1e-12)
    if U.shape[-1] > 5:
        U[..., 5:] = np.maximum(U[..., 5:], 0.0)
    return U


class SubcellFV:
    """HybridSubcellFV (subcell.py:442-950).

    ``coupling="reference"`` reproduces the reference exactly: its DG-FV coupling
    (subcell.py:774-775, 803-805, 836-843) indexes the (E, subcells, nv) arrays with
    boundary-SUBFACE ids, which under JAX gathers are clamped to the last subcell and
    scatters beyond the last subcell are dropped.  ``coupling="subcell"`` uses the subcell
    that owns each subface instead."""

    def __init__(self, op, reconstruction="weno", coupling="reference"):
        self.op, self.mesh, self.gas = op, op.mesh, op.gas
        self.reconstruction = reconstruction
        self.coupling = coupling
        self.ref, self.proj = {}, {}
        for b, block in enumerate(self.mesh.element_blocks):
            rs = RefSubcells(block.element_type)
            self.ref[block.element_type] = rs
            self.proj[block.element_type] = SubcellProjection(op, b, rs)
        self.groups = self._face_groups()

    def _bidx(self, etype, lf):
        return np.flatnonzero(self.ref[etype].boundary_parent == lf).astype(np.int32)

    def _face_groups(self):
        """subcell.py:473-533: owner subfaces per parent face and the neighbour subfaces
        matched by physical subface centre."""
        groups = []
        for ftype, ob, nb, idx in self.op.groups:
            fb = self.mesh.face_blocks[ftype]
            otype = self.mesh.element_blocks[ob].element_type
            osubs, nsubs = [], []
            for f in idx:
                oids = self._bidx(otype, int(fb.owner_face[f]))
                osubs.append(oids)
                if nb >= 0:
                    ntype = self.mesh.element_blocks[nb].element_type
                    nids = self._bidx(ntype, int(fb.neighbor_face[f]))
                    oxyz = self.proj[otype].boundary_centers[int(fb.owner_local[f]), oids]
                    nxyz = self.proj[ntype].boundary_centers[int(fb.neighbor_local[f]), nids]
                    d = np.linalg.norm(oxyz[:, None, :] - nxyz[None, :, :], axis=-1)
                    perm = np.argmin(d, axis=1)
                    scale = max(float(np.max(np.linalg.norm(oxyz, axis=1))), 1.0)
                    if len(np.unique(perm)) != len(oids) or np.max(d[np.arange(len(oids)), perm]) > 2e-6 * scale:
                        raise ValueError(f"Nonconforming subfaces at {ftype} face {f}")
                    nsubs.append(nids[perm])
            groups.append(dict(ftype=ftype, ob=ob, nb=nb, idx=idx, osub=np.asarray(osubs),
                               nsub=None if nb < 0 else np.asarray(nsubs)))
        return groups

    def project(self, states):
        return {k: np.einsum("esi,eiv->esv", self.proj[k].projection, U) for k, U in states.items()}

    def _internal_states(self, name, U):
        """subcell.py:541-665."""
        rs, pj = self.ref[name], self.proj[name]
        own, nbr = rs.internal_owner, rs.internal_neighbor
        if self.reconstruction == "constant":
            return U[:, own], U[:, nbr]
        n, A, vol, cen = pj.internal_normals, pj.internal_areas, pj.volumes, pj.centers
        dU = U[:, nbr] - U[:, own]
        dc = cen[:, nbr] - cen[:, own]
        du_o = np.zeros_like(dU)
        du_n = np.zeros_like(dU)
        for d in range(3):
            contrib = (0.5 * n[:, :, d] * A)[:, :, None] * dU
            g = np.zeros((U.shape[0], rs.count, U.shape[-1]))
            np.add.at(g, (slice(None), own), contrib)
            np.add.at(g, (slice(None), nbr), contrib)
            g = g / np.maximum(vol[:, :, None], 1e-14)
            du_o = du_o + g[:, own] * dc[:, :, d, None]
            du_n = du_n - g[:, nbr] * dc[:, :, d, None]
        with np.errstate(all="ignore"):
            if self.reconstruction == "tvd":
                eps = 1e-12
                ro = dU / (du_o + np.where(du_o >= 0.0, eps, -eps))
                rn = (-dU) / (du_n + np.where(du_n >= 0.0, eps, -eps))
                phio = np.clip(np.where(ro > 0.0, (ro ** 2 + 2 * ro) / (ro ** 2 + ro + 2), 0.0), 0.0, 1.0)
                phin = np.clip(np.where(rn > 0.0, (rn ** 2 + 2 * rn) / (rn ** 2 + rn + 2), 0.0), 0.0, 1.0)
                UL = U[:, own] + 0.5 * phio * du_o
                UR = U[:, nbr] + 0.5 * phin * du_n
            elif self.reconstruction == "weno":
                so, sn = du_o, -du_n
                Phigh = 0.5 * (U[:, own] + U[:, nbr]) + 0.125 * (so - sn)
                Po, Pn = U[:, own] + 0.5 * so, U[:, nbr] - 0.5 * sn
                es = 1e-12
                bh = (sn - so) ** 2 + 0.1 * dU ** 2
                bo = (dU - so) ** 2 + 0.1 * dU ** 2
                bn = (dU - sn) ** 2 + 0.1 * dU ** 2
                bc = dU ** 2
                tau = np.abs(bc - bh)
                d0, d1, d2 = 0.70, 0.28, 0.02
                a0 = d0 * (1.0 + (tau / (bh + es)) ** 2)
                a1 = d1 * (1.0 + (tau / (bo + es)) ** 2)
                a2 = d2 * (1.0 + (tau / (bc + es)) ** 2)
                sa = a0 + a1 + a2
                UL = (a0 / sa) * Phigh + (a1 / sa) * Po + (a2 / sa) * U[:, own]
                a1r = d1 * (1.0 + (tau / (bn + es)) ** 2)
                sr = a0 + a1r + a2
                UR = (a0 / sr) * Phigh + (a1r / sr) * Pn + (a2 / sr) * U[:, nbr]
            else:
                raise ValueError(f"Unknown subcell reconstruction mode: {self.reconstruction!r}")
        return _clamp(UL), _clamp(UR)

    def internal_residual(self, sub):
        """subcell.py:667-688."""
        out = {}
        for name, U in sub.items():
            rs, pj = self.ref[name], self.proj[name]
            UL, UR = self._internal_states(name, U)
            F = self.gas.hllc(UL, UR, pj.internal_normals) * pj.internal_areas[..., None]
            R = np.zeros_like(U)
            np.add.at(R, (slice(None), rs.internal_owner), -F)
            np.add.at(R, (slice(None), rs.internal_neighbor), F)
            out[name] = R
        return out

    def _dg_group_flux(self, states, g, bc):
        """subcell.py:690-746: the DG face flux integrated with the face rule."""
        fb, fm = self.mesh.face_blocks[g["ftype"]], self.op.geo.face[g["ftype"]]
        idx = g["idx"]
        otype = self.mesh.element_blocks[g["ob"]].element_type
        Bo = _basis(otype, self.op.degree, fm.owner_points[idx])
        UL = np.einsum("fqi,fiv->fqv", Bo, states[otype][fb.owner_local[idx]])
        n = fm.normals[idx]
        if g["nb"] >= 0:
            ntype = self.mesh.element_blocks[g["nb"]].element_type
            Bn = _basis(ntype, self.op.degree, fm.neighbor_points[idx])
            UR = np.einsum("fqi,fiv->fqv", Bn, states[ntype][fb.neighbor_local[idx]])
        else:
            UR = UL if bc is None else bc.ghost(UL, n, fb.boundary_tags[idx])
        UL, UR = _clamp(UL), _clamp(UR)
        return np.sum(self.gas.hllc(UL, UR, n) * fm.weights[idx][..., None], axis=1)

    def _gather_scatter(self, etype, subfaces):
        """Subcell indices used to read FV values and to add subface fluxes (-1: dropped)."""
        rs = self.ref[etype]
        if self.coupling == "subcell":
            owner = rs.boundary_owner[subfaces]
            return owner, owner
        return np.clip(subfaces, 0, rs.count - 1), np.where(subfaces < rs.count, subfaces, -1)

    def external_fluxes(self, states, sub, troubled, residual, bc):
        """subcell.py:748-853."""
        new, old = [], []
        for g in self.groups:
            fb = self.mesh.face_blocks[g["ftype"]]
            idx = g["idx"]
            otype = self.mesh.element_blocks[g["ob"]].element_type
            ocells = fb.owner_local[idx]
            pj = self.proj[otype]
            Bo = _basis(otype, self.op.degree, pj.boundary_reference_centers[g["osub"]])
            odg = np.einsum("fki,fiv->fkv", Bo, states[otype][ocells])
            og, osc = self._gather_scatter(otype, g["osub"])
            ofv = sub[otype][ocells[:, None], og]
            oflag = troubled[otype][ocells]
            UL = np.where(oflag[:, None, None], ofv, odg)
            n = pj.boundary_normals[ocells[:, None], g["osub"]]
            A = pj.boundary_areas[ocells[:, None], g["osub"]]
            if g["nb"] >= 0:
                ntype = self.mesh.element_blocks[g["nb"]].element_type
                ncells = fb.neighbor_local[idx]
                Bn = _basis(ntype, self.op.degree, self.proj[ntype].boundary_reference_centers[g["nsub"]])
                ndg = np.einsum("fki,fiv->fkv", Bn, states[ntype][ncells])
                ng, nsc = self._gather_scatter(ntype, g["nsub"])
                nfv = sub[ntype][ncells[:, None], ng]
                nflag = troubled[ntype][ncells]
                UR = np.where(nflag[:, None, None], nfv, ndg)
            else:
                UR = UL if bc is None else bc.ghost(UL, n, fb.boundary_tags[idx])
            UL, UR = _clamp(UL), _clamp(UR)
            F = self.gas.hllc(UL, UR, n) * A[..., None]
            keep = osc >= 0
            rows = np.broadcast_to(ocells[:, None], osc.shape)
            np.add.at(residual[otype], (rows[keep], osc[keep]), -F[keep])
            if g["nb"] >= 0:
                keep = nsc >= 0
                rows = np.broadcast_to(ncells[:, None], nsc.shape)
                np.add.at(residual[ntype], (rows[keep], nsc[keep]), F[keep])
            new.append(F.sum(axis=1))
            old.append(self._dg_group_flux(states, g, bc))
        return new, old

    def recompute(self, states, dg_candidate, dt, troubled, bc=None, additional_rhs=None):
        """subcell.py:855-950."""
        sub = self.project(states)
        res = self.internal_residual(sub)
        new, old = self.external_fluxes(states, sub, troubled, res, bc)
        fv = {k: sub[k] + dt * res[k] / self.proj[k].volumes[..., None] for k in sub}
        if additional_rhs is not None:
            fv = {k: v + dt * np.einsum("esi,eiv->esv", self.proj[k].projection, additional_rhs[k])
                  for k, v in fv.items()}
        rec = {k: subcells_to_dg(v, self.proj[k]) for k, v in fv.items()}
        corrected = {k: v.copy() for k, v in dg_candidate.items()}
        for g, nf, of in zip(self.groups, new, old):
            fb = self.mesh.face_blocks[g["ftype"]]
            idx = g["idx"]
            otype = self.mesh.element_blocks[g["ob"]].element_type
            ocells = fb.owner_local[idx]
            oflag = troubled[otype][ocells]
            if g["nb"] >= 0:
                ntype = self.mesh.element_blocks[g["nb"]].element_type
                ncells = fb.neighbor_local[idx]
                nflag = troubled[ntype][ncells]
            else:
                nflag = np.zeros_like(oflag)
            active = oflag | nflag
            diff = np.where(active[:, None], nf - of, 0.0)
            ovol = self.proj[otype].volumes[ocells].sum(axis=1)
            oc = np.where((active & ~oflag)[:, None], -dt * diff / ovol[:, None], 0.0)
            np.add.at(corrected[otype], ocells, oc[:, None, :])
            if g["nb"] >= 0:
                nvol = self.proj[ntype].volumes[ncells].sum(axis=1)
                nc = np.where((active & ~nflag)[:, None], dt * diff / nvol[:, None], 0.0)
                np.add.at(corrected[ntype], ncells, nc[:, None, :])
        return {k: np.where(troubled[k][:, None, None], rec[k], corrected[k]) for k in states}


class MOODLimiter:
    """HybridMOODSubcellLimiter (limiter.py:267-343)."""

    def __init__(self, op, threshold=5e-2, positivity=None, reconstruction="weno"):
        self.op = op
        self.sensor = TroubledCellSensor(op, threshold)
        self.positivity = PositivityLimiter(op) if positivity is None else positivity
        self.subcell = SubcellFV(op, reconstruction)

    def troubled(self, candidate):
        return mood_troubled(self.op, self.positivity, self.sensor, candidate)

    def recompute(self, base, dg_candidate, dt, bc=None, additional_rhs=None, detection_state=None,
                  troubled_mask=None):
        tr = troubled_mask if troubled_mask is not None else self.troubled(
            dg_candidate if detection_state is None else detection_state)
        if any(np.any(v) for v in tr.values()):
            corrected = self.subcell.recompute(base, dg_candidate, dt, tr, bc, additional_rhs)
        else:
            corrected = dg_candidate
        return self.positivity(corrected)

    def __call__(self, states):
        return self.positivity(states)
