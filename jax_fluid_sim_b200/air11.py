"""Air-11 Park mechanism data: species (molar mass, NASA-7 fits) and 22 reactions.

These are the physical constants of the reference's chemistry
(superboss2300/jax-fluid-sim ``hybrid/chemistry/air11_park.py:10-311``) and must
be identical to them: species order e-, N+, O+, NO+, N2+, O2+, N, O, NO, N2, O2;
NASA-7 coefficient rows [a0..a6] for the low and high temperature ranges; Arrhenius
parameters kf = A T^b exp(-theta/T) in SI units; controlling temperature per
direction ("T", "Ta" = sqrt(T Tv), "Tv"); third-body efficiencies (default 1 for
every species except e-).  ``AIR11_SPECIES`` / ``AIR11_REACTIONS`` are the same
data as ``Species`` / ``Reaction`` records (the reference exports them under these
names, ``hybrid/chemistry/air11_park.py:20,149``).
"""

import numpy as np

from .mechanism import Reaction, Species, make_nasa7, mechanism_tables

R_UNIV = 8.31446261815324      # J / (mol K)
P_STD = 101325.0               # Pa

MW_E = 5.48579909065e-7
MW_N = 0.0140067
MW_O = 0.015999
MW_NO = MW_N + MW_O
MW_N2 = 2.0 * MW_N
MW_O2 = 2.0 * MW_O

SPECIES = ("e-", "N+", "O+", "NO+", "N2+", "O2+", "N", "O", "NO", "N2", "O2")
E, NP, OP, NOP, N2P, O2P, N, O, NO, N2, O2 = range(11)
MOLAR_MASS = np.array([MW_E, MW_N, MW_O, MW_NO, MW_N2, MW_O2, MW_N, MW_O, MW_NO, MW_N2, MW_O2])
CHARGES = (-1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0)
# characteristic vibrational temperatures of the diatomic species (0: not diatomic); only
# the two-temperature relaxation reads them
THETA_V = (0.0, 0.0, 0.0, 3380.0, 3160.0, 2700.0, 0.0, 0.0, 2740.0, 3395.0, 2270.0)

# (t_low, t_mid, t_high, low coefficients, high coefficients)
NASA7 = (
    (298.15, 1000.0, 6000.0, (2.5, 0.0, 0.0, 0.0, 0.0, -745.375, -11.7208122),
     (2.5, 0.0, 0.0, 0.0, 0.0, -745.375, -11.7208122)),
    (298.15, 1000.0, 6000.0,
     (2.79781357, -1.41287178e-03, 2.68686998e-06, -2.31615591e-09, 7.49585578e-13, 225548.731, 3.59928845),
     (2.51210704, 1.75367440e-06, -1.50557538e-08, 7.06834189e-12, -6.31861166e-16, 225597.004, 4.92236293)),
    (298.15, 1000.0, 6000.0, (2.5, 0.0, 0.0, 0.0, 0.0, 187935.284, 4.39337676),
     (2.48542028, 2.56978695e-05, -1.28833378e-08, 1.65525487e-12, 1.09933344e-16, 187940.874, 4.47425446)),
    (298.15, 1000.0, 6000.0,
     (3.69301231, -1.34229158e-03, 2.67343395e-06, -1.02609308e-09, -6.95610492e-14, 118103.055, 3.09126691),
     (2.94587702, 1.40325260e-03, -4.95503196e-07, 7.95948973e-11, -4.72076668e-15, 118244.340, 6.70644634)),
    (298.15, 1000.0, 6000.0,
     (3.77540711, -2.06459157e-03, 4.75752301e-06, -3.15664228e-09, 6.70509973e-13, 180481.115, 2.69322178),
     (3.58661363, 2.53071949e-04, 1.84778214e-07, -4.55257223e-11, 3.26818029e-15, 180390.994, 3.09584143)),
    (298.15, 1000.0, 6000.0,
     (4.61017167, -6.35951952e-03, 1.42425624e-05, -1.20997923e-08, 3.70956878e-12, 139742.229, -0.201326941),
     (3.31675922, 1.11522244e-03, -3.83492556e-07, 5.72784687e-11, -2.77648381e-15, 139876.823, 5.44726469)),
    (200.0, 1000.0, 6000.0, (2.5, 0.0, 0.0, 0.0, 0.0, 56104.638, 4.1939088),
     (2.4159429, 1.74890650e-04, -1.19023690e-07, 3.02262440e-11, -2.03609830e-15, 56133.775, 4.6496095)),
    (200.0, 1000.0, 6000.0,
     (3.16826710, -3.27931884e-03, 6.64306396e-06, -6.12806624e-09, 2.11265971e-12, 29122.2592, 2.05193346),
     (2.54363697, -2.73162486e-05, -4.19029520e-09, 4.95481845e-12, -4.79553694e-16, 29226.012, 4.92229457)),
    (200.0, 1000.0, 6000.0,
     (4.21859896, -4.63988124e-03, 1.10443049e-05, -9.34055507e-09, 2.80554874e-12, 9845.09964, 2.28061001),
     (3.26071234, 1.19101135e-03, -4.29122646e-07, 6.94481463e-11, -4.03295681e-15, 9921.43132, 6.36900518)),
    (200.0, 1000.0, 6000.0,
     (3.53100528, -1.23660988e-04, -5.02999433e-07, 2.43530612e-09, -1.40881235e-12, -1046.97628, 2.96747038),
     (2.95257637, 1.39690040e-03, -4.92631603e-07, 7.86010195e-11, -4.60755204e-15, -923.948688, 5.87188762)),
    (200.0, 1000.0, 6000.0,
     (3.78245636, -2.99673416e-03, 9.84730201e-06, -9.68129509e-09, 3.24372837e-12, -1063.94356, 3.65767573),
     (3.66096065, 6.56365811e-04, -1.41149627e-07, 2.05797935e-11, -1.29913436e-15, -1215.97718, 3.41536279)),
)

# (reactants, products, A, b, theta, third_body, efficiencies, forward T, reverse T)
REACTIONS = (
    (((N2, 1),), ((N, 2),), 7.0e15, -1.6, 113200.0, True, ((O, 4.285714285714286), (N, 4.285714285714286)), "Ta", "T"),
    (((N2, 1), (E, 1)), ((N, 2), (E, 1)), 3.0e18, -1.6, 113200.0, False, (), "Tv", "Tv"),
    (((O2, 1),), ((O, 2),), 2.0e15, -1.5, 59360.0, True, ((O, 5.0), (N, 5.0)), "Ta", "T"),
    (((NO, 1),), ((N, 1), (O, 1)), 5.0e9, 0.0, 75500.0, True,
     ((NO, 22.0), (N, 22.0), (O, 22.0), (NP, 22.0), (OP, 22.0)), "Ta", "T"),
    (((N2, 1), (O, 1)), ((NO, 1), (N, 1)), 5.7e6, 0.42, 42938.0, False, (), "T", "T"),
    (((NO, 1), (O, 1)), ((O2, 1), (N, 1)), 8.4e6, 0.0, 19400.0, False, (), "T", "T"),
    (((N, 1), (O, 1)), ((NOP, 1), (E, 1)), 5.3e6, 0.0, 31900.0, False, (), "T", "Tv"),
    (((O, 2),), ((O2P, 1), (E, 1)), 7.1e-4, 2.7, 80600.0, False, (), "T", "Tv"),
    (((N, 2),), ((N2P, 1), (E, 1)), 4.4e1, 1.5, 67500.0, False, (), "T", "Tv"),
    (((NOP, 1), (O, 1)), ((NP, 1), (O2, 1)), 1.0e6, 0.5, 77200.0, False, (), "T", "T"),
    (((NP, 1), (N2, 1)), ((N2P, 1), (N, 1)), 1.0e6, 0.5, 12200.0, False, (), "T", "T"),
    (((O2P, 1), (N, 1)), ((NP, 1), (O2, 1)), 8.7e7, 0.14, 28600.0, False, (), "T", "T"),
    (((OP, 1), (NO, 1)), ((NP, 1), (O2, 1)), 1.4e-1, 1.9, 26600.0, False, (), "T", "T"),
    (((O2P, 1), (N2, 1)), ((N2P, 1), (O2, 1)), 9.9e6, 0.0, 40700.0, False, (), "T", "T"),
    (((O2P, 1), (O, 1)), ((OP, 1), (O2, 1)), 4.0e6, 0.09, 18000.0, False, (), "T", "T"),
    (((NOP, 1), (N, 1)), ((OP, 1), (N2, 1)), 3.4e7, -1.08, 12800.0, False, (), "T", "T"),
    (((NOP, 1), (O2, 1)), ((O2P, 1), (NO, 1)), 2.4e7, 0.41, 32600.0, False, (), "T", "T"),
    (((NOP, 1), (O, 1)), ((O2P, 1), (N, 1)), 7.2e6, 0.29, 48600.0, False, (), "T", "T"),
    (((OP, 1), (N2, 1)), ((N2P, 1), (O, 1)), 9.1e5, 0.36, 22800.0, False, (), "T", "T"),
    (((NOP, 1), (N, 1)), ((N2P, 1), (O, 1)), 7.2e7, 0.0, 35500.0, False, (), "T", "T"),
    (((O, 1), (E, 1)), ((OP, 1), (E, 2)), 3.9e27, -3.78, 158500.0, False, (), "Tv", "T"),
    (((N, 1), (E, 1)), ((NP, 1), (E, 2)), 2.5e28, -3.82, 168200.0, False, (), "Tv", "T"),
)


def _species():
    return tuple(Species(name, molar_mass=float(w), charge=q, poly=make_nasa7(*fit), is_diatomic=tv > 0.0,
                         theta_v=tv)
                 for name, w, q, fit, tv in zip(SPECIES, MOLAR_MASS, CHARGES, NASA7, THETA_V))


def _reactions():
    return tuple(Reaction(reactants=reac, products=prod, A=a, b=bb, theta=th, third_body=tb, efficiencies=eff,
                          fwd_temp=ft, rev_temp=rt)
                 for reac, prod, a, bb, th, tb, eff, ft, rt in REACTIONS)


AIR11_SPECIES = _species()
AIR11_REACTIONS = _reactions()


def tables():
    """Dense arrays of the Air-11 mechanism (``mechanism_tables`` layout)."""
    return mechanism_tables(AIR11_SPECIES, AIR11_REACTIONS)
