"""Reaction-mechanism description: species, reactions and NASA-7 fits as plain data.

The reference's ``hybrid/chemistry/mechanism.py:26-123`` and ``nasa.py:18-44`` describe a
mechanism with frozen dataclasses (``Species``, ``Reaction``, ``NASAPolynomial``); the same
constructors are kept here so that a mechanism written for the reference builds
unchanged.  ``mechanism_tables`` turns one into the dense arrays that the chemistry
kernels take (``dgb_chem_mechanism``): stoichiometry nu' and nu'', third-body efficiencies
(default 1 for every species except one named ``e-``, ``mechanism.py:103-114``),
Arrhenius parameters, temperature modes and NASA-7 ranges and coefficients.
"""

from dataclasses import dataclass

import numpy as np

TEMPERATURE_MODES = {"T": 0, "Ta": 1, "Tv": 2}


@dataclass(frozen=True)
class NASAPolynomial:
    t_low: float
    t_mid: float
    t_high: float
    coeffs_low: tuple
    coeffs_high: tuple


def make_nasa7(t_low, t_mid, t_high, low, high):
    if len(low) != 7 or len(high) != 7:
        raise ValueError("NASA-7 polynomials take 7 coefficients per range")
    return NASAPolynomial(float(t_low), float(t_mid), float(t_high), tuple(float(a) for a in low),
                          tuple(float(a) for a in high))


@dataclass(frozen=True)
class Species:
    name: str
    molar_mass: float
    charge: float = 0.0
    poly: NASAPolynomial | None = None
    is_diatomic: bool = False
    theta_v: float = 0.0


@dataclass(frozen=True)
class Reaction:
    reactants: tuple
    products: tuple
    A: float
    b: float
    theta: float
    third_body: bool = False
    efficiencies: tuple = ()
    reversible: bool = True      # not read by the rate law (mechanism.py:159-220 ignores it too)
    fwd_temp: str = "T"
    rev_temp: str = "T"


def mechanism_tables(species, reactions):
    """Dense float64/int32 arrays of a mechanism (the layout of ``dgb_chem_mechanism``)."""
    ns, nr = len(species), len(reactions)
    nu_f = np.zeros((nr, ns))
    nu_r = np.zeros((nr, ns))
    alpha = np.zeros((nr, ns))
    A, b, theta = np.zeros(nr), np.zeros(nr), np.zeros(nr)
    third = np.zeros(nr, np.int32)
    fmode = np.zeros(nr, np.int32)
    rmode = np.zeros(nr, np.int32)
    for r, rx in enumerate(reactions):
        for s, c in rx.reactants:
            nu_f[r, s] += float(c)
        for s, c in rx.products:
            nu_r[r, s] += float(c)
        A[r], b[r], theta[r] = rx.A, rx.b, rx.theta
        third[r] = int(bool(rx.third_body))
        fmode[r], rmode[r] = TEMPERATURE_MODES[rx.fwd_temp], TEMPERATURE_MODES[rx.rev_temp]
        if rx.third_body:
            for s, sp in enumerate(species):
                if sp.name != "e-":
                    alpha[r, s] = 1.0
            for s, e in rx.efficiencies:
                alpha[r, s] = e
    if any(sp.poly is None for sp in species):
        raise ValueError("every species needs a NASA-7 polynomial")
    trange = np.array([[sp.poly.t_low, sp.poly.t_mid, sp.poly.t_high] for sp in species])
    coeffs = np.array([[sp.poly.coeffs_low, sp.poly.coeffs_high] for sp in species])
    molar_mass = np.array([sp.molar_mass for sp in species], dtype=np.float64)
    return dict(nu_f=nu_f, nu_r=nu_r, alpha=alpha, A=A, b=b, theta=theta, third=third, fmode=fmode, rmode=rmode,
                trange=trange, coeffs=coeffs, molar_mass=molar_mass)
