"""Pointwise physics: EOS, Euler fluxes, HLLC/Rusanov, viscous flux, boundary ghosts.

Oracle restatement of ``hybrid/solver.py:63-406`` (WALE omitted: off in every
workload) and ``hybrid/boundary.py:6-102``.
"""

import numpy as np

RHO_FLOOR = 1.0e-14


class Gas:
    """solver.py:20-61 constructor constants."""

    def __init__(self, gamma=1.4, gas_constant=1.0, dynamic_viscosity=0.0, prandtl=0.72, n_species=0):
        self.gamma = float(gamma)
        self.R = float(gas_constant)
        self.mu = float(dynamic_viscosity)
        self.prandtl = float(prandtl)
        self.cp = self.gamma * self.R / (self.gamma - 1.0)
        self.kappa = self.mu * self.cp / self.prandtl
        self.n_species = int(n_species)
        self.nvars = 5 + self.n_species

    # solver.py:63-81
    def to_conserved(self, W):
        rho = W[..., 0]
        vel = W[..., 1:4]
        E = W[..., 4] / (self.gamma - 1.0) + 0.5 * rho * np.sum(vel ** 2, axis=-1)
        parts = [rho[..., None], rho[..., None] * vel, E[..., None]]
        if self.n_species:
            parts.append(rho[..., None] * W[..., 5:])
        return np.concatenate(parts, axis=-1)

    # solver.py:83-98
    def to_primitive(self, U):
        rho = U[..., 0]
        m = U[..., 1:4]
        srho = np.maximum(rho, RHO_FLOOR)
        vel = m / srho[..., None]
        ke = 0.5 * np.sum(m ** 2, axis=-1) / srho
        p = (self.gamma - 1.0) * (U[..., 4] - ke)
        parts = [rho[..., None], vel, p[..., None]]
        if self.n_species:
            parts.append(U[..., 5:] / srho[..., None])
        return np.concatenate(parts, axis=-1)

    # solver.py:100-122
    def normal_flux(self, U, n):
        W = self.to_primitive(U)
        rho, vel, p = W[..., 0], W[..., 1:4], W[..., 4]
        un = np.sum(vel * n, axis=-1)
        parts = [(rho * un)[..., None], rho[..., None] * vel * un[..., None] + p[..., None] * n,
                 (un * (U[..., 4] + p))[..., None]]
        if self.n_species:
            parts.append(U[..., 5:] * un[..., None])
        return np.concatenate(parts, axis=-1)

    # solver.py:124-130
    def flux_tensor(self, U):
        eye = np.eye(3)
        return np.stack([self.normal_flux(U, eye[d]) for d in range(3)], axis=-2)

    # solver.py:132-152
    def rusanov(self, UL, UR, n):
        WL, WR = self.to_primitive(UL), self.to_primitive(UR)
        unl = np.sum(WL[..., 1:4] * n, axis=-1)
        unr = np.sum(WR[..., 1:4] * n, axis=-1)
        cl = np.sqrt(self.gamma * np.maximum(WL[..., 4], 0.0) / np.maximum(WL[..., 0], RHO_FLOOR))
        cr = np.sqrt(self.gamma * np.maximum(WR[..., 4], 0.0) / np.maximum(WR[..., 0], RHO_FLOOR))
        smax = np.maximum(np.abs(unl) + cl, np.abs(unr) + cr)
        return 0.5 * (self.normal_flux(UL, n) + self.normal_flux(UR, n)) - 0.5 * smax[..., None] * (UR - UL)

    @staticmethod
    def _safe(v, tol=1.0e-14):
        """solver.py:154-161."""
        return np.where(np.abs(v) > tol, v, np.where(v >= 0.0, tol, -tol))

    def _star(self, U, W, s, sm, n):
        """solver.py:209-243."""
        rho, vel, p = W[..., 0], W[..., 1:4], W[..., 4]
        un = np.sum(vel * n, axis=-1)
        den = self._safe(s - sm)
        comp = (s - un) / den
        rho_s = rho * comp
        vel_s = vel + (sm - un)[..., None] * n
        p_s = p + rho * (s - un) * (sm - un)
        E_s = ((s - un) * U[..., 4] - p * un + p_s * sm) / den
        parts = [rho_s[..., None], rho_s[..., None] * vel_s, E_s[..., None]]
        if self.n_species:
            parts.append(U[..., 5:] * comp[..., None])
        return np.concatenate(parts, axis=-1)

    def hllc(self, UL, UR, n):
        """solver.py:163-207 (wave speeds) and :245-300 (flux, fallback, identical-state)."""
        with np.errstate(all="ignore"):
            WL, WR = self.to_primitive(UL), self.to_primitive(UR)
            FL, FR = self.normal_flux(UL, n), self.normal_flux(UR, n)
            rl, rr = WL[..., 0], WR[..., 0]
            pl, pr = WL[..., 4], WR[..., 4]
            unl = np.sum(WL[..., 1:4] * n, axis=-1)
            unr = np.sum(WR[..., 1:4] * n, axis=-1)
            cl = np.sqrt(np.maximum(self.gamma * pl / np.maximum(rl, RHO_FLOOR), 0.0))
            cr = np.sqrt(np.maximum(self.gamma * pr / np.maximum(rr, RHO_FLOOR), 0.0))
            sl = np.minimum(unl - cl, unr - cr)
            sr = np.maximum(unl + cl, unr + cr)
            den = rl * (sl - unl) - rr * (sr - unr)
            sm = (pr - pl + rl * unl * (sl - unl) - rr * unr * (sr - unr)) / self._safe(den)
            FsL = FL + sl[..., None] * (self._star(UL, WL, sl, sm, n) - UL)
            FsR = FR + sr[..., None] * (self._star(UR, WR, sr, sm, n) - UR)
            h = np.where((sl >= 0.0)[..., None], FL,
                         np.where((sm >= 0.0)[..., None], FsL,
                                  np.where((sr > 0.0)[..., None], FsR, FR)))
            valid = (rl > 0.0) & (rr > 0.0) & (pl > 0.0) & (pr > 0.0) & np.all(np.isfinite(h), axis=-1)
            robust = np.where(valid[..., None], h, self.rusanov(UL, UR, n))
            same = np.all(UL == UR, axis=-1)
            return np.where(same[..., None], FL, robust)

    # solver.py:307-315
    def viscous_variables(self, U):
        W = self.to_primitive(U)
        T = W[..., 4] / (np.maximum(W[..., 0], RHO_FLOOR) * self.R)
        return np.concatenate([W[..., 1:4], T[..., None]], axis=-1)

    # solver.py:357-406 (constant mu, kappa)
    def viscous_flux(self, U, grad):
        W = self.to_primitive(U)
        vel = W[..., 1:4]
        G = grad[..., 0:3, :]
        gT = grad[..., 3, :]
        div = np.trace(G, axis1=-2, axis2=-1)
        stress = self.mu * (G + np.swapaxes(G, -1, -2) - (2.0 / 3.0) * div[..., None, None] * np.eye(3))
        out = np.zeros(U.shape[:-1] + (3, self.nvars))
        out[..., :, 1:4] = np.swapaxes(stress, -1, -2)
        out[..., :, 4] = np.einsum("...i,...id->...d", vel, stress) + self.kappa * gT
        return out


class FarfieldWallBoundary:
    """boundary.py:6-102.  Tags resolved from the mesh's physical names."""

    def __init__(self, gas, physical_names, farfield_primitive, inlet_names=("inlet",),
                 outlet_names=("outlet",),
                 wall_names=("walls", "sphere_wall", "cylinder_wall", "airfoil_wall", "symmetry"),
                 no_slip_names=("sphere_wall", "cylinder_wall", "airfoil_wall"),
                 slip_names=("walls", "symmetry"), wall_temperature=None):
        self.gas = gas
        self.farfield = np.asarray(farfield_primitive, np.float64)
        self.wall_temperature = None if wall_temperature is None else float(wall_temperature)

        def tags(names):
            return np.asarray([physical_names[n] for n in names if n in physical_names], np.int64)

        self.inlet_tags, self.outlet_tags = tags(inlet_names), tags(outlet_names)
        self.wall_tags, self.no_slip_tags, self.slip_tags = tags(wall_names), tags(no_slip_names), tags(slip_names)

    @staticmethod
    def matches(t, choices):
        if choices.size == 0:
            return np.zeros(np.shape(t), bool)
        return np.any(np.asarray(t)[..., None] == choices, axis=-1)

    def ghost(self, U, n, t):
        """boundary.py:54-72: slip-reflect on walls, far-field on inlets, copy elsewhere."""
        W = self.gas.to_primitive(U)
        wall = self.matches(t, self.wall_tags)[:, None, None]
        vel = W[..., 1:4]
        un = np.sum(vel * n, axis=-1)
        Ww = W.copy()
        Ww[..., 1:4] = vel - 2.0 * un[..., None] * n
        G = np.where(wall, Ww, W)
        inlet = self.matches(t, self.inlet_tags)[:, None, None]
        G = np.where(inlet, np.broadcast_to(self.farfield, W.shape), G)
        return self.gas.to_conserved(G)

    def viscous_ghost(self, U, n, t):
        """boundary.py:74-102."""
        v = self.gas.viscous_variables(U)
        g = v
        ns = self.matches(t, self.no_slip_tags)[:, None, None]
        nsv = v.copy()
        nsv[..., 0:3] = -v[..., 0:3]
        if self.wall_temperature is not None:
            nsv[..., 3] = 2.0 * self.wall_temperature - v[..., 3]
        g = np.where(ns, nsv, g)
        slip = self.matches(t, self.slip_tags)[:, None, None]
        vel = v[..., 0:3]
        un = np.sum(vel * n, axis=-1)
        sv = v.copy()
        sv[..., 0:3] = vel - 2.0 * un[..., None] * n
        g = np.where(slip, sv, g)
        inlet = self.matches(t, self.inlet_tags)[:, None, None]
        ff = self.gas.viscous_variables(self.gas.to_conserved(np.broadcast_to(self.farfield, U.shape)))
        return np.where(inlet, ff, g)
