"""DG operators and SSP-RK3: the residual-and-update path on the CPU.

Oracle restatement of
* ``hybrid/spatial.py:20-45,47-72,137-249``   anchor-form Euler residual and rhs;
* ``hybrid/navier_stokes.py:27-352``           BR2 viscous residual and rhs;
* ``hybrid/time_integration.py:49-169``        characteristic lengths, stable_dt;
* ``hybrid/time_integration.py:264-312,404-583`` stage blend, admissibility, checked_step;
* ``hybrid/limiter.py:11-185,267-343``         positivity limiter, sensor, MOOD.
"""

import numpy as np

from .elements import basis as _basis
from .geometry import Geometry
from .physics import Gas


class Operator:
    """HybridEulerOperator + HybridNavierStokesOperator (spatial.py, navier_stokes.py)."""

    def __init__(self, mesh, gas: Gas, degree, br2_stabilization=None):
        self.mesh = mesh
        self.gas = gas
        self.degree = degree
        self.geo = Geometry(mesh, degree)
        self.br2 = float((degree + 1) * (degree + 2) / 2 if br2_stabilization is None else br2_stabilization)
        self.groups = []
        for ftype, fb in mesh.face_blocks.items():                      # spatial.py:20-39
            keys = sorted({(int(o), int(n)) for o, n in zip(fb.owner_block, fb.neighbor_block)})
            for ob, nb in keys:
                idx = np.flatnonzero((fb.owner_block == ob) & (fb.neighbor_block == nb))
                self.groups.append((ftype, ob, nb, idx))

    def names(self):
        return [b.element_type for b in self.mesh.element_blocks]

    def _side_basis(self, ftype, block_id, idx, side):
        fm = self.geo.face[ftype]
        pts = (fm.owner_points if side == 0 else fm.neighbor_points)[idx]
        etype = self.mesh.element_blocks[block_id].element_type
        return _basis(etype, self.degree, pts)

    # ---------------- Euler (spatial.py) ----------------
    def residual(self, states, bc=None):
        g = self.gas
        anchors = {k: U[:, 0, :] for k, U in states.items()}            # spatial.py:41-45
        res = {}
        for b, block in enumerate(self.mesh.element_blocks):            # spatial.py:47-72
            ref, m = self.geo.ref[block.element_type], self.geo.element[b]
            U, a = states[block.element_type], anchors[block.element_type]
            Uq = a[:, None, :] + np.einsum("qi,eiv->eqv", ref.B, U - a[:, None, :])
            F = g.flux_tensor(Uq) - g.flux_tensor(a)[:, None, :, :]
            res[block.element_type] = np.einsum("eqid,eqdv,eq->eiv", m.grad, F, m.wdet)
        for ftype, ob, nb, idx in self.groups:                           # spatial.py:142-232
            fb, fm = self.mesh.face_blocks[ftype], self.geo.face[ftype]
            otype = self.mesh.element_blocks[ob].element_type
            ocells = fb.owner_local[idx]
            Bo = self._side_basis(ftype, ob, idx, 0)
            ao = anchors[otype][ocells]
            Uo = ao[:, None, :] + np.einsum("fqi,fiv->fqv", Bo, states[otype][ocells] - ao[:, None, :])
            n = fm.normals[idx]
            w = fm.weights[idx]
            if nb >= 0:
                ntype = self.mesh.element_blocks[nb].element_type
                ncells = fb.neighbor_local[idx]
                Bn = self._side_basis(ftype, nb, idx, 1)
                an = anchors[ntype][ncells]
                Un = an[:, None, :] + np.einsum("fqi,fiv->fqv", Bn, states[ntype][ncells] - an[:, None, :])
            else:
                Un = Uo if bc is None else bc.ghost(Uo, n, fb.boundary_tags[idx])
            Fh = g.hllc(Uo, Un, n)
            wo = (Fh - g.normal_flux(ao[:, None, :], n)) * w[..., None]
            np.add.at(res[otype], ocells, -np.einsum("fqi,fqv->fiv", Bo, wo))
            if nb >= 0:
                wn = (Fh - g.normal_flux(an[:, None, :], n)) * w[..., None]
                np.add.at(res[ntype], ncells, np.einsum("fqi,fqv->fiv", Bn, wn))
        return res

    def apply_inverse_mass(self, res):
        return {b.element_type: np.einsum("eij,ejv->eiv", self.geo.element[k].minv, res[b.element_type])
                for k, b in enumerate(self.mesh.element_blocks)}

    def inviscid_rhs(self, states, bc=None):
        return self.apply_inverse_mass(self.residual(states, bc))

    # ---------------- BR2 viscous (navier_stokes.py) ----------------
    def _trace(self, states, group, bc):
        """navier_stokes.py:27-110."""
        g = self.gas
        ftype, ob, nb, idx = group
        fb, fm = self.mesh.face_blocks[ftype], self.geo.face[ftype]
        d = {"idx": idx, "ftype": ftype, "ob": ob, "nb": nb}
        otype = self.mesh.element_blocks[ob].element_type
        d["ocells"] = fb.owner_local[idx]
        d["Bo"] = self._side_basis(ftype, ob, idx, 0)
        Uon = states[otype][d["ocells"]]
        d["Uo"] = np.einsum("fqi,fiv->fqv", d["Bo"], Uon)
        d["von"] = g.viscous_variables(Uon)
        vo = np.einsum("fqi,fim->fqm", d["Bo"], d["von"])
        n = fm.normals[idx]
        if nb >= 0:
            ntype = self.mesh.element_blocks[nb].element_type
            d["ncells"] = fb.neighbor_local[idx]
            d["Bn"] = self._side_basis(ftype, nb, idx, 1)
            Unn = states[ntype][d["ncells"]]
            d["Un"] = np.einsum("fqi,fiv->fqv", d["Bn"], Unn)
            d["vnn"] = g.viscous_variables(Unn)
            vn = np.einsum("fqi,fim->fqm", d["Bn"], d["vnn"])
        else:
            t = fb.boundary_tags[idx]
            d["Un"] = d["Uo"] if bc is None else bc.ghost(d["Uo"], n, t)
            vn = g.viscous_variables(d["Un"]) if bc is None else bc.viscous_ghost(d["Uo"], n, t)
        d["jump"] = vn - vo
        return d

    def _br2(self, states, bc):
        """navier_stokes.py:138-208."""
        lift = {b.element_type: np.zeros(states[b.element_type].shape[:2] + (4, 3)) for b in self.mesh.element_blocks}
        data = []
        for group in self.groups:
            d = self._trace(states, group, bc)
            fm = self.geo.face[d["ftype"]]
            w, n = fm.weights[d["idx"]], fm.normals[d["idx"]]
            otype = self.mesh.element_blocks[d["ob"]].element_type
            rhs_o = 0.5 * np.einsum("fq,fqm,fqd,fqi->fimd", w, d["jump"], n, d["Bo"])
            d["lo"] = np.einsum("fij,fjmd->fimd", self.geo.element[d["ob"]].minv[d["ocells"]], rhs_o)
            np.add.at(lift[otype], d["ocells"], d["lo"])
            if d["nb"] >= 0:
                ntype = self.mesh.element_blocks[d["nb"]].element_type
                rhs_n = 0.5 * np.einsum("fq,fqm,fqd,fqi->fimd", w, d["jump"], n, d["Bn"])
                d["ln"] = np.einsum("fij,fjmd->fimd", self.geo.element[d["nb"]].minv[d["ncells"]], rhs_n)
                np.add.at(lift[ntype], d["ncells"], d["ln"])
            data.append(d)
        vol_grad = {}
        for b, block in enumerate(self.mesh.element_blocks):
            ref, m = self.geo.ref[block.element_type], self.geo.element[b]
            v = self.gas.viscous_variables(states[block.element_type])
            raw = np.einsum("eim,eqid->eqmd", v, m.grad)
            vol_grad[block.element_type] = raw + np.einsum("qi,eimd->eqmd", ref.B, lift[block.element_type])
        return vol_grad, data

    def viscous_residual(self, states, bc=None):
        """navier_stokes.py:210-324."""
        g = self.gas
        vol_grad, data = self._br2(states, bc)
        res = {}
        for b, block in enumerate(self.mesh.element_blocks):
            ref, m = self.geo.ref[block.element_type], self.geo.element[b]
            Uq = np.einsum("qi,eiv->eqv", ref.B, states[block.element_type])
            F = g.viscous_flux(Uq, vol_grad[block.element_type])
            res[block.element_type] = -np.einsum("eqid,eqdv,eq->eiv", m.grad, F, m.wdet)
        for d in data:
            fb, fm = self.mesh.face_blocks[d["ftype"]], self.geo.face[d["ftype"]]
            idx = d["idx"]
            n, w = fm.normals[idx], fm.weights[idx]
            go = self.geo.physical_basis_gradients(d["ob"], d["ocells"], fm.owner_points[idx])
            raw_o = np.einsum("fim,fqid->fqmd", d["von"], go)
            grad_o = raw_o + self.br2 * np.einsum("fqi,fimd->fqmd", d["Bo"], d["lo"])
            Fo = g.viscous_flux(d["Uo"], grad_o)
            if d["nb"] >= 0:
                gn = self.geo.physical_basis_gradients(d["nb"], d["ncells"], fm.neighbor_points[idx])
                raw_n = np.einsum("fim,fqid->fqmd", d["vnn"], gn)
                grad_n = raw_n + self.br2 * np.einsum("fqi,fimd->fqmd", d["Bn"], d["ln"])
                Fface = 0.5 * (Fo + g.viscous_flux(d["Un"], grad_n))
            else:
                Fface = Fo
            Fn = np.einsum("fqdv,fqd->fqv", Fface, n)
            if d["nb"] < 0 and bc is not None:
                wall = bc.matches(fb.boundary_tags[idx], bc.wall_tags)
                Fn[..., 4] = np.where(wall[:, None], 0.0, Fn[..., 4])
            W = Fn * w[..., None]
            otype = self.mesh.element_blocks[d["ob"]].element_type
            np.add.at(res[otype], d["ocells"], np.einsum("fqi,fqv->fiv", d["Bo"], W))
            if d["nb"] >= 0:
                ntype = self.mesh.element_blocks[d["nb"]].element_type
                np.add.at(res[ntype], d["ncells"], -np.einsum("fqi,fqv->fiv", d["Bn"], W))
        return res

    def viscous_rhs(self, states, bc=None):
        return self.apply_inverse_mass(self.viscous_residual(states, bc))

    def rhs(self, states, bc=None):
        """navier_stokes.py:338-343."""
        e = self.inviscid_rhs(states, bc)
        if self.gas.mu == 0.0:
            return e
        v = self.viscous_rhs(states, bc)
        return {k: e[k] + v[k] for k in e}

    # ---------------- limiter support (limiter.py:28-92) ----------------
    def face_sample_basis(self):
        pts = {b.element_type: [] for b in self.mesh.element_blocks}
        for ftype, ob, nb, idx in self.groups:
            fm = self.geo.face[ftype]
            pts[self.mesh.element_blocks[ob].element_type].append(fm.owner_points[idx].reshape(-1, 3))
            if nb >= 0:
                pts[self.mesh.element_blocks[nb].element_type].append(fm.neighbor_points[idx].reshape(-1, 3))
        out = {}
        for t, chunks in pts.items():
            if chunks:
                uniq = np.unique(np.round(np.concatenate(chunks), decimals=12), axis=0)
                out[t] = _basis(t, self.degree, uniq)
            else:
                out[t] = np.zeros((0, len(self.geo.ref[t].nodes)))
        return out

    def cell_mean(self, b, U):
        ref, m = self.geo.ref[self.mesh.element_blocks[b].element_type], self.geo.element[b]
        Uq = np.einsum("qi,eiv->eqv", ref.B, U)
        return np.einsum("eqv,eq->ev", Uq, m.wdet) / m.wdet.sum(axis=1)[:, None]


class TimeIntegrator:
    """HybridSSPRK3 (time_integration.py) with optional limiter objects below."""

    def __init__(self, op: Operator, cfl=0.15, limiter=None, density_floor=1e-7, pressure_floor=1e-7):
        self.op, self.cfl, self.limiter = op, float(cfl), limiter
        self.density_floor, self.pressure_floor = float(density_floor), float(pressure_floor)
        self.lengths = self._lengths()

    def _lengths(self):
        """time_integration.py:49-91."""
        mesh, geo = self.op.mesh, self.op.geo
        sums = {b.element_type: np.zeros(len(b.connectivity)) for b in mesh.element_blocks}
        for ftype, fb in mesh.face_blocks.items():
            area = geo.face[ftype].weights.sum(axis=1)
            for k, b in enumerate(mesh.element_blocks):
                o = np.flatnonzero(fb.owner_block == k)
                np.add.at(sums[b.element_type], fb.owner_local[o], area[o])
                n = np.flatnonzero(fb.neighbor_block == k)
                np.add.at(sums[b.element_type], fb.neighbor_local[n], area[n])
        out = {}
        for k, b in enumerate(mesh.element_blocks):
            vol = geo.element[k].wdet.sum(axis=1)
            out[b.element_type] = np.maximum(2.0 * vol / sums[b.element_type],
                                             0.25 * vol ** (1.0 / 3.0) / (self.op.degree + 1))
        return out

    def stable_dt(self, states):
        """time_integration.py:93-169 (WALE off)."""
        g, P = self.op.gas, self.op.degree
        df = 2 * P + 1
        rates = []
        for b in self.op.mesh.element_blocks:
            W = g.to_primitive(states[b.element_type])
            rho = np.maximum(W[..., 0], 1e-14)
            p = np.maximum(W[..., 4], 1e-14)
            speed = np.linalg.norm(W[..., 1:4], axis=-1) + np.sqrt(g.gamma * p / rho)
            h = self.lengths[b.element_type]
            rate = df * speed.max(axis=1) / h
            if g.mu > 0.0:
                rmin = np.maximum(rho.mean(axis=1), 0.1)
                diff = np.maximum((4.0 / 3.0) * g.mu / rmin, g.kappa / (rmin * g.cp))
                rate = rate + 2.0 * self.op.br2 * df ** 2 * diff / np.maximum(h, 0.01) ** 2
            rates.append(np.max(np.nan_to_num(rate, nan=1e7, posinf=1e7)))
        return float(np.clip(self.cfl / max(max(rates), 1e-12), 1e-7, 1e-3))

    def admissibility(self, states):
        """time_integration.py:291-312."""
        g = self.op.gas
        finite, rmins, pmins = True, [], []
        for U in states.values():
            finite = finite and bool(np.all(np.isfinite(U)))
            rho = U[..., 0]
            rmins.append(np.min(rho))
            ke = 0.5 * np.sum(U[..., 1:4] ** 2, axis=-1) / np.maximum(rho, 1e-14)
            pmins.append(np.min((g.gamma - 1.0) * (U[..., 4] - ke)))
        rmin, pmin = float(min(rmins)), float(min(pmins))
        return bool(finite and rmin >= self.density_floor and pmin >= self.pressure_floor), rmin, pmin

    def _limit(self, states):
        return states if self.limiter is None else self.limiter(states)

    def rk_stage(self, base, cur, dt, alpha, beta, bc=None):
        """time_integration.py:404-439."""
        mood = self.limiter is not None and hasattr(self.limiter, "recompute")
        if mood:
            inv = self.op.inviscid_rhs(cur, bc)
            visc = self.op.viscous_rhs(cur, bc)
            total = {k: inv[k] + visc[k] for k in inv}
        else:
            total = self.op.rhs(cur, bc)
            visc = None
        euler = {k: cur[k] + dt * total[k] for k in cur}
        unlimited = {k: alpha * base[k] + beta * euler[k] for k in cur}
        if mood:
            rec = self.limiter.recompute(cur, euler, dt, bc, visc, detection_state=unlimited)
            result = self.limiter.positivity({k: alpha * base[k] + beta * rec[k] for k in cur})
        else:
            result = self._limit(unlimited)
        return (result,) + self.admissibility(result)

    def checked_step(self, states, dt, bc=None):
        """time_integration.py:441-583: three stages; non-MOOD returns the AND/min of the
        three admissibility checks, MOOD returns the last stage's."""
        mood = self.limiter is not None and hasattr(self.limiter, "recompute")
        s1, v1, r1, p1 = self.rk_stage(states, states, dt, 0.0, 1.0, bc)
        s2, v2, r2, p2 = self.rk_stage(states, s1, dt, 0.75, 0.25, bc)
        s3, v3, r3, p3 = self.rk_stage(states, s2, dt, 1.0 / 3.0, 2.0 / 3.0, bc)
        if mood:
            return s3, v3, r3, p3
        return s3, v1 and v2 and v3, min(r1, r2, r3), min(p1, p2, p3)


class PositivityLimiter:
    """limiter.py:11-147."""

    def __init__(self, op: Operator, density_floor=1e-10, pressure_floor=1e-10, relative_floor=0.05):
        self.op = op
        self.density_floor, self.pressure_floor = float(density_floor), float(pressure_floor)
        self.relative_floor = float(relative_floor)
        self.face_basis = op.face_sample_basis()

    def sample(self, etype, U):
        ref = self.op.geo.ref[etype]
        return np.concatenate([U, np.einsum("qi,eiv->eqv", ref.B, U),
                               np.einsum("qi,eiv->eqv", self.face_basis[etype], U)], axis=1)

    def _pressure_ok(self, mean, dev, theta, floor):
        s = mean[:, None, :] + theta[:, None, None] * dev
        return np.min(self.op.gas.to_primitive(s)[..., 4], axis=1) >= floor

    def limit_block(self, b, U):
        etype = self.op.mesh.element_blocks[b].element_type
        mean = self.op.cell_mean(b, U)
        Wm = self.op.gas.to_primitive(mean)
        rfloor = np.maximum(self.density_floor, self.relative_floor * Wm[:, 0])
        pfloor = np.maximum(self.pressure_floor, self.relative_floor * Wm[:, 4])
        s = self.sample(etype, U)
        dev = s - mean[:, None, :]
        rmin = s[..., 0].min(axis=1)
        with np.errstate(all="ignore"):
            dtheta = np.where(rmin < rfloor, (mean[:, 0] - rfloor) / np.maximum(mean[:, 0] - rmin, 1e-30), 1.0)
            upper = np.clip(dtheta, 0.0, 1.0)
            lo, hi = np.zeros_like(upper), upper.copy()
            for _ in range(30):
                mid = 0.5 * (lo + hi)
                ok = self._pressure_ok(mean, dev, mid, pfloor)
                lo, hi = np.where(ok, mid, lo), np.where(ok, hi, mid)
            theta = np.where(self._pressure_ok(mean, dev, upper, pfloor), upper, lo)
        return mean[:, None, :] + theta[:, None, None] * (U - mean[:, None, :])

    def __call__(self, states):
        return {b.element_type: self.limit_block(k, states[b.element_type])
                for k, b in enumerate(self.op.mesh.element_blocks)}


class TroubledCellSensor:
    """limiter.py:150-185."""

    def __init__(self, op: Operator, threshold=5e-2):
        self.op, self.threshold = op, float(threshold)
        self.proj = {}
        if op.degree >= 2:
            for t, ref in op.geo.ref.items():
                p1 = _basis(t, 1, ref.nodes)
                self.proj[t] = p1 @ np.linalg.pinv(p1)

    def block_sensor(self, etype, U):
        if self.op.degree < 2:
            return np.zeros(U.shape[0])
        W = self.op.gas.to_primitive(U)[..., [0, 4]]
        low = np.einsum("ij,ejm->eim", self.proj[etype], W)
        ratio = np.sum((W - low) ** 2, axis=1) / np.maximum(np.sum(W ** 2, axis=1), 1e-12)
        return ratio.max(axis=-1)

    def __call__(self, states):
        s = {k: self.block_sensor(k, U) for k, U in states.items()}
        return s, {k: v > self.threshold for k, v in s.items()}


def mood_troubled(op: Operator, positivity: PositivityLimiter, sensor: TroubledCellSensor, candidate):
    """limiter.py:285-300: sensor flags OR non-finite / below-floor samples (nodes, volume and
    face points, cell mean)."""
    _, flags = sensor(candidate)
    out = {}
    for k, b in enumerate(op.mesh.element_blocks):
        name = b.element_type
        s = positivity.sample(name, candidate[name])
        s = np.concatenate([s, op.cell_mean(k, candidate[name])[:, None, :]], axis=1)
        W = op.gas.to_primitive(s)
        with np.errstate(invalid="ignore"):
            bad = (~np.all(np.isfinite(W), axis=(1, 2)) | (W[..., 0].min(axis=1) < positivity.density_floor)
                   | (W[..., 4].min(axis=1) < positivity.pressure_floor))
        out[name] = flags[name] | bad
    return out
