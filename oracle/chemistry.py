"""Finite-rate Air-11 chemistry on the CPU (oracle).

Restatement of ``hybrid/chemistry/nasa.py:47-118`` (NASA-7 fits with the
temperature clamped to each species' range), ``mechanism.py:125-287`` (forward
rates, Gibbs equilibrium constants, mass-action net rates with third bodies and
the mass-conserving correction, T(e) Newton inversion), ``integrator.py:31-104``
(point-implicit Newton on rho - rho0 - dt w(rho, T) with T re-derived from the
initial internal energy after every update) and ``coupling.py:116-197`` (per-node
coupling with the dimensionless scaling).  The reference differentiates the
residual with JAX; here the Jacobian is written out analytically, with JAX's
convention for the derivative of max/min/clip at a tie (half to each side), and is
pinned to the reference's forward-mode Jacobian in the golden fixtures.

Test infrastructure: only the tests, the smoke check and the CPU baseline of the
benchmark use this module.  The mechanism's constants are the data
tables of ``jax_fluid_sim_b200/air11.py``.
"""

import numpy as np

from jax_fluid_sim_b200.air11 import P_STD, R_UNIV, tables

CLIP_EXP, MIN_KC, MIN_C = 700.0, 1.0e-300, 1.0e-100


class Mechanism:
    """mechanism.py:58-220 over the dense tables of ``mechanism_tables`` (Air-11 by default)."""

    def __init__(self, table=None):
        t = tables() if table is None else table
        for k, v in t.items():
            setattr(self, k, v)
        self.dnu = self.nu_r - self.nu_f
        self.dn = self.dnu.sum(axis=1)
        self.ns = len(self.molar_mass)

    # nasa.py:56-118 -> per-species (cp/R, h/RT, s/R) at T clamped to each range
    def _coeffs(self, T):
        Tc = np.clip(T, self.trange[:, 0], self.trange[:, 2])
        a = np.where((Tc < self.trange[:, 1])[:, None], self.coeffs[:, 0], self.coeffs[:, 1])
        return Tc, a

    def cp_R(self, T):
        Tc, a = self._coeffs(T)
        return a[:, 0] + a[:, 1] * Tc + a[:, 2] * Tc ** 2 + a[:, 3] * Tc ** 3 + a[:, 4] * Tc ** 4

    def h_RT(self, T):
        Tc, a = self._coeffs(T)
        return (a[:, 0] + a[:, 1] * Tc / 2.0 + a[:, 2] * Tc ** 2 / 3.0 + a[:, 3] * Tc ** 3 / 4.0
                + a[:, 4] * Tc ** 4 / 5.0 + a[:, 5] / Tc)

    def s_R(self, T):
        Tc, a = self._coeffs(T)
        return (a[:, 0] * np.log(Tc) + a[:, 1] * Tc + a[:, 2] * Tc ** 2 / 2.0 + a[:, 3] * Tc ** 3 / 3.0
                + a[:, 4] * Tc ** 4 / 4.0 + a[:, 6])

    def select(self, mode, T, Tv):
        """mechanism.py:125-128."""
        Ta = np.sqrt(max(T * Tv, 1.0))
        return np.where(mode == 1, Ta, np.where(mode == 2, Tv, T))

    def kf(self, T, Tv):
        Te = np.maximum(self.select(self.fmode, T, Tv), 10.0)
        return self.A * Te ** self.b * np.exp(-self.theta / Te)

    def Kc(self, T, Tv):
        Te = np.maximum(self.select(self.rmode, T, Tv), 10.0)
        out = np.empty(len(Te))
        for r, t in enumerate(Te):
            g = self.h_RT(t) - self.s_R(t)
            dG = float(self.dnu[r] @ g)
            out[r] = np.exp(-np.clip(dG, -CLIP_EXP, CLIP_EXP)) * (P_STD / (R_UNIV * t)) ** self.dn[r]
        return out

    def rates(self, rho, T, Tv=None, jacobian=False):
        """mechanism.py:159-220: (omega_dot, w_dot[, d w_dot / d rho])."""
        Tv = T if Tv is None else Tv
        W = self.molar_mass
        Craw = rho / W
        C = np.maximum(Craw, 0.0)
        kf = self.kf(T, Tv)
        kr = kf / np.maximum(self.Kc(T, Tv), MIN_KC)
        logC = np.log(np.maximum(C, MIN_C))
        lf, lr = self.nu_f @ logC, self.nu_r @ logC
        fwd = np.exp(np.clip(lf, -CLIP_EXP, CLIP_EXP))
        rev = np.exp(np.clip(lr, -CLIP_EXP, CLIP_EXP))
        Meff = self.alpha @ C
        coll = np.where(self.third == 1, Meff, 1.0)
        qnet = (kf * fwd - kr * rev) * coll
        omega = self.dnu.T @ qnet
        wd = omega * W
        S = max(rho.sum(), 1.0e-14)
        Y = np.maximum(rho, 0.0) / S
        sw = wd.sum()
        wfix = wd - Y * sw
        if not jacobian:
            return omega, wfix
        # d C_s / d rho_s through max(rho/W, 0): JAX's rule splits the derivative evenly
        # at a tie, so a species clamped to exactly zero keeps half of 1/W.
        # d log C / d rho is zero below MIN_C; clips pass the derivative inside the range.
        dC = np.where(Craw > 0.0, 1.0, np.where(Craw == 0.0, 0.5, 0.0)) / W
        dlog = np.where(C > MIN_C, 1.0, np.where(C == MIN_C, 0.5, 0.0)) * dC / np.maximum(C, MIN_C)
        okf = np.where(np.abs(lf) < CLIP_EXP, 1.0, np.where(np.abs(lf) == CLIP_EXP, 0.5, 0.0))
        okr = np.where(np.abs(lr) < CLIP_EXP, 1.0, np.where(np.abs(lr) == CLIP_EXP, 0.5, 0.0))
        dfwd = (fwd * okf)[:, None] * self.nu_f * dlog[None, :]
        drev = (rev * okr)[:, None] * self.nu_r * dlog[None, :]
        dq = (kf[:, None] * dfwd - kr[:, None] * drev) * coll[:, None]
        dcoll = np.where((self.third == 1)[:, None], self.alpha * dC[None, :], 0.0)
        dq += ((kf * fwd - kr * rev))[:, None] * dcoll
        dwd = W[:, None] * (self.dnu.T @ dq)                   # [s][j]
        dS = 1.0 if rho.sum() > 1.0e-14 else (0.5 if rho.sum() == 1.0e-14 else 0.0)
        dmax = np.where(rho > 0.0, 1.0, np.where(rho == 0.0, 0.5, 0.0))
        dY = np.diag(dmax / S) - (np.maximum(rho, 0.0) / S ** 2)[:, None] * dS
        J = dwd - dY * sw - Y[:, None] * dwd.sum(axis=0)[None, :]
        return omega, wfix, J

    def e_cv(self, T):
        """Per-species internal energy e_s and cv_s in J/kg at T."""
        W = self.molar_mass
        e = (self.h_RT(T) - 1.0) * (R_UNIV * T / W)
        cv = (self.cp_R(T) - 1.0) * (R_UNIV / W)
        return e, cv

    def internal_energy(self, rho, T):
        """mixture_properties()['internal_energy'] (mechanism.py:222-260)."""
        Y = np.maximum(rho, 0.0) / max(rho.sum(), 1.0e-14)
        return float(Y @ self.e_cv(T)[0])

    def temperature(self, rho, e_target, T_init=1000.0, num_iters=10):
        """mechanism.py:262-287."""
        Y = np.maximum(rho, 0.0) / max(rho.sum(), 1.0e-14)
        T = float(T_init)
        for _ in range(num_iters):
            Ts = min(max(T, 50.0), 50000.0)
            e, cv = self.e_cv(Ts)
            res = float(Y @ e) - e_target
            dT = -res / max(float(Y @ cv), 1.0e-5)
            T = min(max(T + min(max(dT, -0.5 * T), 0.5 * T), 100.0), 50000.0)
        return T


def implicit_step(mech, rho_species, T, dt, max_newton_iters=16, constant_temperature=True):
    """integrator.py:31-104."""
    rho0 = np.maximum(rho_species, 1.0e-20)
    total = rho0.sum()
    e_init = mech.internal_energy(rho0, T)
    rho, Tk = rho0.copy(), float(T)
    I = np.eye(mech.ns)
    for _ in range(max_newton_iters):
        _, w, J = mech.rates(rho, Tk, jacobian=True)
        res = rho - rho0 - dt * w
        d = np.linalg.solve(I - dt * J, -res)
        rho = np.maximum(rho + d, 0.0)
        if not constant_temperature:
            Tk = mech.temperature(rho, e_init, T_init=Tk)
    return rho * (total / rho.sum()), Tk


class Coupler:
    """ReactingFlowCoupler (coupling.py:19-209), single temperature."""

    def __init__(self, max_newton_iters=12, dimensionless=False, reference_temperature=300.0,
                 reference_pressure=101325.0, reference_length=1.0, gamma=1.4):
        self.mech = Mechanism()
        self.iters = max_newton_iters
        self.dimensionless = dimensionless
        self.gamma = gamma
        self.T_ref, self.p_ref, self.L_ref = reference_temperature, reference_pressure, reference_length
        mean_mw = 1.0 / (0.767 / (2.0 * 0.0140067) + 0.233 / (2.0 * 0.015999))
        self.R_ref = R_UNIV / mean_mw
        self.rho_ref = self.p_ref / (self.R_ref * self.T_ref)
        self.u_ref = float(np.sqrt(self.R_ref * self.T_ref))
        self.e_ref = self.u_ref ** 2
        self.t_ref = self.L_ref / self.u_ref

    def react_node(self, u, dt):
        """coupling.py:116-177."""
        ns = self.mech.ns
        rho_t = max(u[0], 1.0e-14)
        rs = np.maximum(u[5:5 + ns], 0.0)
        rs = rs * (rho_t / max(rs.sum(), 1.0e-20))
        ek = 0.5 * float(np.sum(u[1:4] ** 2)) / rho_t ** 2
        if self.dimensionless:
            es = max(u[4] / rho_t - ek, 1.0e-4)
            e = es * self.e_ref
            rp = rs * self.rho_ref
            Tg = max((self.gamma - 1.0) * es * self.T_ref, 200.0)
            T0 = self.mech.temperature(rp, e, T_init=Tg, num_iters=8)
            new, _ = implicit_step(self.mech, rp, T0, dt * self.t_ref, self.iters, constant_temperature=False)
            new = new / self.rho_ref
        else:
            e = max(u[4] / rho_t - ek, 1.0e3)
            T0 = self.mech.temperature(rs, e, T_init=1000.0, num_iters=8)
            new, _ = implicit_step(self.mech, rs, T0, dt, self.iters, constant_temperature=False)
        new = np.maximum(new, 0.0)
        new = new * (rho_t / max(new.sum(), 1.0e-20))
        out = u.copy()
        out[5:5 + ns] = new
        return out

    def react_block(self, U, dt):
        """coupling.py:179-197 for a scalar dt."""
        out = np.empty_like(U)
        for e in range(U.shape[0]):
            for n in range(U.shape[1]):
                out[e, n] = self.react_node(U[e, n], dt)
        return out


# ----------------------------------------------------------------------------------------------
# The same restatement over many nodes at once (numpy batches): rows of rho are nodes.  Every
# element-wise step is the per-node one above; only the sums run in numpy's batched order.

def _batch_coeffs(mech, T):
    """nasa.py:56-118 for T of shape (N,): Tc (N, ns) and the coefficient rows (N, ns, 7)."""
    Tc = np.clip(T[:, None], mech.trange[:, 0], mech.trange[:, 2])
    a = np.where((Tc < mech.trange[:, 1])[..., None], mech.coeffs[:, 0], mech.coeffs[:, 1])
    return Tc, a


def _batch_h_RT(mech, T):
    Tc, a = _batch_coeffs(mech, T)
    return (a[..., 0] + a[..., 1] * Tc / 2.0 + a[..., 2] * Tc ** 2 / 3.0 + a[..., 3] * Tc ** 3 / 4.0
            + a[..., 4] * Tc ** 4 / 5.0 + a[..., 5] / Tc)


def _batch_g_RT(mech, T):
    Tc, a = _batch_coeffs(mech, T)
    h = (a[..., 0] + a[..., 1] * Tc / 2.0 + a[..., 2] * Tc ** 2 / 3.0 + a[..., 3] * Tc ** 3 / 4.0
         + a[..., 4] * Tc ** 4 / 5.0 + a[..., 5] / Tc)
    s = (a[..., 0] * np.log(Tc) + a[..., 1] * Tc + a[..., 2] * Tc ** 2 / 2.0 + a[..., 3] * Tc ** 3 / 3.0
         + a[..., 4] * Tc ** 4 / 4.0 + a[..., 6])
    return h - s


def _batch_e_cv(mech, T):
    Tc, a = _batch_coeffs(mech, T)
    W = mech.molar_mass
    h = (a[..., 0] + a[..., 1] * Tc / 2.0 + a[..., 2] * Tc ** 2 / 3.0 + a[..., 3] * Tc ** 3 / 4.0
         + a[..., 4] * Tc ** 4 / 5.0 + a[..., 5] / Tc)
    cp = a[..., 0] + a[..., 1] * Tc + a[..., 2] * Tc ** 2 + a[..., 3] * Tc ** 3 + a[..., 4] * Tc ** 4
    return (h - 1.0) * (R_UNIV * T[:, None] / W), (cp - 1.0) * (R_UNIV / W)


def batch_rates(mech, rho, T):
    """Mechanism.rates(..., jacobian=True) for rho (N, ns), T (N,) with Tv = T: (w_dot, J)."""
    W = mech.molar_mass
    Craw = rho / W
    C = np.maximum(Craw, 0.0)
    # controlling temperatures (mechanism.py:125-128) with Tv = T: mode 1 is sqrt(max(T T, 1))
    T1 = np.sqrt(np.maximum(T * T, 1.0))
    Tf = np.maximum(np.where(mech.fmode[None, :] == 1, T1[:, None], T[:, None]), 10.0)     # (N, nr)
    Tr = np.maximum(np.where(mech.rmode[None, :] == 1, T1[:, None], T[:, None]), 10.0)
    kf = mech.A * Tf ** mech.b * np.exp(-mech.theta / Tf)
    g0 = _batch_g_RT(mech, np.maximum(T, 10.0))
    g1 = _batch_g_RT(mech, np.maximum(T1, 10.0))
    g = np.where((mech.rmode == 1)[None, :, None], g1[:, None, :], g0[:, None, :])        # (N, nr, ns)
    dG = np.einsum("nrs,rs->nr", g, mech.dnu)
    Kc = np.exp(-np.clip(dG, -CLIP_EXP, CLIP_EXP)) * (P_STD / (R_UNIV * Tr)) ** mech.dn
    kr = kf / np.maximum(Kc, MIN_KC)
    logC = np.log(np.maximum(C, MIN_C))
    lf, lr = logC @ mech.nu_f.T, logC @ mech.nu_r.T
    fwd = np.exp(np.clip(lf, -CLIP_EXP, CLIP_EXP))
    rev = np.exp(np.clip(lr, -CLIP_EXP, CLIP_EXP))
    Meff = C @ mech.alpha.T
    coll = np.where(mech.third[None, :] == 1, Meff, 1.0)
    qnet = (kf * fwd - kr * rev) * coll
    omega = qnet @ mech.dnu
    wd = omega * W
    Sraw = rho.sum(axis=1)
    S = np.maximum(Sraw, 1.0e-14)
    Y = np.maximum(rho, 0.0) / S[:, None]
    sw = wd.sum(axis=1)
    wfix = wd - Y * sw[:, None]
    dC = np.where(Craw > 0.0, 1.0, np.where(Craw == 0.0, 0.5, 0.0)) / W
    dlog = np.where(C > MIN_C, 1.0, np.where(C == MIN_C, 0.5, 0.0)) * dC / np.maximum(C, MIN_C)
    okf = np.where(np.abs(lf) < CLIP_EXP, 1.0, np.where(np.abs(lf) == CLIP_EXP, 0.5, 0.0))
    okr = np.where(np.abs(lr) < CLIP_EXP, 1.0, np.where(np.abs(lr) == CLIP_EXP, 0.5, 0.0))
    dfwd = (fwd * okf)[..., None] * mech.nu_f[None] * dlog[:, None, :]
    drev = (rev * okr)[..., None] * mech.nu_r[None] * dlog[:, None, :]
    dq = (kf[..., None] * dfwd - kr[..., None] * drev) * coll[..., None]
    dcoll = np.where((mech.third == 1)[:, None], mech.alpha, 0.0)[None] * dC[:, None, :]
    dq += (kf * fwd - kr * rev)[..., None] * dcoll
    dwd = W[None, :, None] * np.einsum("rs,nrj->nsj", mech.dnu, dq)
    dS = np.where(Sraw > 1.0e-14, 1.0, np.where(Sraw == 1.0e-14, 0.5, 0.0))
    dmax = np.where(rho > 0.0, 1.0, np.where(rho == 0.0, 0.5, 0.0))
    eye = np.eye(mech.ns)
    dY = (eye[None] * (dmax / S[:, None])[:, :, None]
          - (np.maximum(rho, 0.0) / (S ** 2)[:, None])[:, :, None] * dS[:, None, None])
    J = dwd - dY * sw[:, None, None] - Y[:, :, None] * dwd.sum(axis=1)[:, None, :]
    return wfix, J


def batch_temperature(mech, rho, e_target, T_init, num_iters=10):
    """Mechanism.temperature for rows of rho."""
    S = np.maximum(rho.sum(axis=1), 1.0e-14)
    Y = np.maximum(rho, 0.0) / S[:, None]
    T = np.asarray(T_init, np.float64).copy()
    for _ in range(num_iters):
        Ts = np.minimum(np.maximum(T, 50.0), 50000.0)
        e, cv = _batch_e_cv(mech, Ts)
        res = (Y * e).sum(axis=1) - e_target
        dT = -res / np.maximum((Y * cv).sum(axis=1), 1.0e-5)
        T = np.minimum(np.maximum(T + np.minimum(np.maximum(dT, -0.5 * T), 0.5 * T), 100.0), 50000.0)
    return T


def batch_implicit_step(mech, rho_species, T, dt, max_newton_iters):
    """implicit_step(..., constant_temperature=False) for rows of rho_species."""
    rho0 = np.maximum(rho_species, 1.0e-20)
    total = rho0.sum(axis=1)
    S0 = np.maximum(total, 1.0e-14)
    e_init = (np.maximum(rho0, 0.0) / S0[:, None] * _batch_e_cv(mech, T)[0]).sum(axis=1)
    rho, Tk = rho0.copy(), T.copy()
    I = np.eye(mech.ns)[None]
    for _ in range(max_newton_iters):
        w, J = batch_rates(mech, rho, Tk)
        res = rho - rho0 - dt * w
        d = np.linalg.solve(I - dt * J, -res[..., None])[..., 0]
        rho = np.maximum(rho + d, 0.0)
        Tk = batch_temperature(mech, rho, e_init, Tk)
    return rho * (total / rho.sum(axis=1))[:, None]


def batch_react_block(coupler, U, dt):
    """Coupler.react_block over all nodes at once (coupling.py:116-197, scalar dt)."""
    mech, ns = coupler.mech, coupler.mech.ns
    u = U.reshape(-1, U.shape[-1])
    rho_t = np.maximum(u[:, 0], 1.0e-14)
    rs = np.maximum(u[:, 5:5 + ns], 0.0)
    rs = rs * (rho_t / np.maximum(rs.sum(axis=1), 1.0e-20))[:, None]
    ek = 0.5 * np.sum(u[:, 1:4] ** 2, axis=1) / rho_t ** 2
    if coupler.dimensionless:
        es = np.maximum(u[:, 4] / rho_t - ek, 1.0e-4)
        rp = rs * coupler.rho_ref
        Tg = np.maximum((coupler.gamma - 1.0) * es * coupler.T_ref, 200.0)
        T0 = batch_temperature(mech, rp, es * coupler.e_ref, Tg, num_iters=8)
        new = batch_implicit_step(mech, rp, T0, dt * coupler.t_ref, coupler.iters) / coupler.rho_ref
    else:
        e = np.maximum(u[:, 4] / rho_t - ek, 1.0e3)
        T0 = batch_temperature(mech, rs, e, np.full(len(u), 1000.0), num_iters=8)
        new = batch_implicit_step(mech, rs, T0, dt, coupler.iters)
    new = np.maximum(new, 0.0)
    new = new * (rho_t / np.maximum(new.sum(axis=1), 1.0e-20))[:, None]
    out = u.copy()
    out[:, 5:5 + ns] = new
    return out.reshape(U.shape)
