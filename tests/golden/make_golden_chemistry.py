"""Golden fixtures of the reference's Air-11 chemistry (run in the build container).

    python tests/golden/make_golden_chemistry.py [/path/to/reference]

Runs ``hybrid/chemistry`` of the reference under the numpy stand-in for JAX
(``jax.jacobian`` there is forward-mode differentiation with dual numbers) and
stores rates, temperature inversion,
the point-implicit step and the coupler's block update in
``tests/golden/chemistry.npz``.
"""

import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REFERENCE = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
sys.path.insert(0, str(HERE / "refshim"))
_pkg = types.ModuleType("hybrid")
_pkg.__path__ = [str(REFERENCE / "hybrid")]
sys.modules["hybrid"] = _pkg

import jax  # noqa: E402
import jax.numpy as jnp  # noqa: E402
from hybrid.chemistry.air11_park import Air11ParkMechanism  # noqa: E402
from hybrid.chemistry.coupling import ReactingFlowCoupler  # noqa: E402
from hybrid.chemistry.integrator import PointImplicitIntegrator  # noqa: E402
from hybrid.chemistry.mechanism import Reaction, ReactionMechanism, Species  # noqa: E402
from hybrid.chemistry.nasa import make_nasa7  # noqa: E402

# The 3-species H2/O2 mechanism of the reference's extensibility test
# (tests/test_air11_chemistry.py:132-172): NASA-7 rows, molar masses, one reaction.
ROCKET_NASA = (
    ((3.298, 8.249e-4, -8.143e-7, -9.475e-11, 4.134e-13, -1012.5, -3.294),
     (2.932, 8.266e-4, -1.464e-7, 1.541e-11, -6.888e-16, -813.0, -1.024)),
    ((3.782, -2.996e-3, 9.847e-6, -9.681e-9, 3.243e-12, -1063.9, 3.657),
     (3.660, 6.563e-4, -1.411e-7, 2.057e-11, -1.299e-15, -1215.9, 3.415)),
    ((4.198, -2.036e-3, 6.520e-6, -5.487e-9, 1.771e-12, -30293.7, -0.849),
     (2.677, 2.973e-3, -7.737e-7, 9.443e-11, -4.269e-15, -29885.8, 6.882)),
)
ROCKET_MW = (0.002016, 0.031998, 0.018015)


def rocket(out):
    species = [Species(n, molar_mass=w, poly=make_nasa7(200.0, 1000.0, 6000.0, list(lo), list(hi)))
               for n, w, (lo, hi) in zip(("H2", "O2", "H2O"), ROCKET_MW, ROCKET_NASA)]
    mech = ReactionMechanism(species, [Reaction(reactants=((0, 2), (1, 1)), products=((2, 2),), A=1.0e11, b=0.0,
                                                theta=15000.0, reversible=True)])
    states = [np.array([0.2, 0.8, 0.01]), np.array([0.05, 0.3, 0.6]), np.array([0.1, 0.0, 0.4])]
    temps = [800.0, 2000.0, 3500.0]
    om, wd, jac = [], [], []
    for s in states:
        for T in temps:
            o, w = mech.net_production_rates(jnp.asarray(s), jnp.asarray(T))
            om.append(np.asarray(o))
            wd.append(np.asarray(w))
            jac.append(np.asarray(jax.jacobian(lambda r: mech.net_production_rates(r, jnp.asarray(T))[1])(
                jnp.asarray(s))))
    out["rocket_nasa"] = np.asarray(ROCKET_NASA)
    out["rocket_mw"] = np.asarray(ROCKET_MW)
    out["rocket_states"] = np.asarray(states)
    out["rocket_temps"] = np.asarray(temps)
    out["rocket_omega"] = np.asarray(om)
    out["rocket_wdot"] = np.asarray(wd)
    out["rocket_jac"] = np.asarray(jac)


def main():
    out = {}
    mech = Air11ParkMechanism()
    states = [
        np.array([0, 0, 0, 0, 0, 0, 0, 0, 0, 0.79, 0.21], float),
        np.array([1e-6, 1e-5, 1e-5, 1e-4, 1e-5, 1e-5, 0.2, 0.1, 0.05, 0.4, 0.1]),
        np.array([1e-4, 0.05, 0.05, 0.05, 0.02, 0.02, 0.3, 0.2, 0.01, 0.1, 0.05]),
        np.array([0, 0, 0, 0, 0, 0, 0, 0, 0, 0.8, 0.4], float),
    ]
    temps = [500.0, 3000.0, 8000.0, 15000.0]
    rates_w, rates_o = [], []
    for s in states:
        for T in temps:
            o, w = mech.net_production_rates(jnp.asarray(s), jnp.asarray(T))
            rates_o.append(np.asarray(o))
            rates_w.append(np.asarray(w))
    out["rate_states"] = np.asarray(states)
    out["rate_temps"] = np.asarray(temps)
    out["rate_omega"] = np.asarray(rates_o)
    out["rate_wdot"] = np.asarray(rates_w)
    # d w_dot / d rho by the stand-in's forward-mode jacobian (what integrator.py:78 uses),
    # at the rate states and at a state with species clamped to exactly zero
    jac_states = states + [np.array([0, 0.01, 0, 0.2, 0, 0, 0.3, 0.2, 0, 0.4, 0.0])]
    jacs = []
    for s in jac_states:
        for T in temps:
            jacs.append(np.asarray(jax.jacobian(
                lambda r: mech.net_production_rates(r, jnp.asarray(T))[1])(jnp.asarray(s))))
    out["jac_states"] = np.asarray(jac_states)
    out["jac_wdot"] = np.asarray(jacs)
    # temperature inversion (mechanism.py:262-287)
    comp = np.zeros(11)
    comp[9], comp[10] = 0.767, 0.233
    inv_T = []
    for T in (500.0, 1500.0, 4000.0, 8000.0):
        e = float(mech.mixture_properties(jnp.asarray(comp), jnp.asarray(T))["internal_energy"])
        inv_T.append([T, e, float(mech.recover_temperature_from_energy(jnp.asarray(comp), e, T_init=1000.0))])
    out["inversion"] = np.asarray(inv_T)
    # point-implicit step (the reference's own test case), constant and coupled temperature
    integ = PointImplicitIntegrator(mech, max_newton_iters=16, tolerance=1.0e-7)
    rho0 = np.zeros(11)
    rho0[9], rho0[10] = 0.8, 0.4
    r1, _, _ = integ.step(jnp.asarray(rho0), jnp.asarray(8000.0), dt=1.0e-6, constant_temperature=True)
    r2, T2, _ = integ.step(jnp.asarray(rho0), jnp.asarray(8000.0), dt=1.0e-6, constant_temperature=False)
    out["step_rho0"] = rho0
    out["step_const"] = np.asarray(r1)
    out["step_coupled"] = np.asarray(r2)
    out["step_coupled_T"] = np.asarray(T2)
    # coupler, SI (the reference test state) and dimensionless (Mach-8 sphere scaling)
    coupler = ReactingFlowCoupler(mech, max_newton_iters=16)
    rho, u, T = 1.2, 2000.0, 6000.0
    Y = np.zeros(11)
    Y[9], Y[10] = 0.767, 0.233
    e_th = float(mech.mixture_properties(jnp.asarray(rho * Y), jnp.asarray(T))["internal_energy"])
    node = np.zeros(16)
    node[0], node[1], node[4], node[5:] = rho, rho * u, rho * (e_th + 0.5 * u * u), rho * Y
    rng = np.random.default_rng(5)
    U = np.broadcast_to(node, (2, 3, 16)).copy()
    U[..., 4] *= 1.0 + 0.05 * rng.random((2, 3))
    out["coupler_U"] = U
    out["coupler_dt"] = np.asarray(1.0e-7)
    out["coupler_out"] = np.asarray(coupler.react_block(jnp.asarray(U), 1.0e-7))
    # at dt = 1e-7 the 16 Newton iterations of this state oscillate without converging, so
    # the result depends on round-off; at dt = 1e-9 they converge to machine precision
    out["coupler_conv_dt"] = np.asarray(1.0e-9)
    out["coupler_conv_out"] = np.asarray(coupler.react_block(jnp.asarray(U), 1.0e-9))
    dimless = ReactingFlowCoupler(mech, dimensionless=True, reference_temperature=220.0, reference_pressure=500.0,
                                  reference_length=0.1)
    Ud = np.zeros((2, 3, 16))
    Ud[..., 0] = 1.0 + 3.0 * rng.random((2, 3))
    vel = 8.0 * np.sqrt(1.4) * (0.2 + 0.1 * rng.random((2, 3)))
    Ud[..., 1] = Ud[..., 0] * vel
    pres = 1.0 + 80.0 * rng.random((2, 3))
    Ud[..., 4] = pres / 0.4 + 0.5 * Ud[..., 0] * vel ** 2
    Ud[..., 5 + 9] = 0.767 * Ud[..., 0]
    Ud[..., 5 + 10] = 0.233 * Ud[..., 0]
    out["dimless_U"] = Ud
    out["dimless_dt"] = np.asarray(2.0e-3)
    out["dimless_out"] = np.asarray(dimless.react_block(jnp.asarray(Ud), 2.0e-3))
    rocket(out)
    np.savez_compressed(HERE / "chemistry.npz", **out)
    print("wrote chemistry.npz")


if __name__ == "__main__":
    main()
