"""GPU chemistry (dgb_react_block, dgb_chem_rates) against the reference fixtures and the oracle.

Tolerances: rates and their Jacobian to 1e-12 of the largest entry (float64 evaluation
order only); the coupler's species to 1e-10 of the node density for the converged SI
state and 2e-5 for the dimensionless Mach-8 state, where I - dt J has condition numbers
near 1e12 and the reference and the oracle already differ by 7e-6.
"""

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle.chemistry import Coupler, Mechanism

GOLDEN = np.load(Path(__file__).resolve().parent / "golden" / "chemistry.npz")

pytestmark = pytest.mark.gpu


def _cuda(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.fixture(scope="module")
def mech():
    from jax_fluid_sim_b200 import Air11ParkMechanism
    return Air11ParkMechanism()


def _close(a, b, tol):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.max(np.abs(b)), 1e-300)
    assert np.max(np.abs(a - b)) <= tol * scale, (np.max(np.abs(a - b)) / scale)


def test_rates_and_jacobian_match_reference(mech):
    states, temps = GOLDEN["rate_states"], GOLDEN["rate_temps"]
    rho = np.repeat(states, len(temps), axis=0)
    T = np.tile(temps, len(states))
    omega, wdot = mech.net_production_rates(_cuda(rho), _cuda(T))
    for k in range(len(rho)):
        _close(omega[k].cpu(), GOLDEN["rate_omega"][k], 1e-12)
        _close(wdot[k].cpu(), GOLDEN["rate_wdot"][k], 1e-12)
    js = GOLDEN["jac_states"]
    J = mech.production_rate_jacobian(_cuda(np.repeat(js, len(temps), axis=0)), _cuda(np.tile(temps, len(js))))
    for k in range(len(js) * len(temps)):
        _close(J[k].cpu(), GOLDEN["jac_wdot"][k], 1e-12)


def test_mass_conservation_and_benchmark(mech):
    """tests/test_air11_chemistry.py:40-86 on the GPU rates."""
    rho = np.zeros((1, 11))
    rho[0, 9], rho[0, 10] = 0.8, 0.4
    omega, _ = mech.net_production_rates(_cuda(rho), _cuda([8000.0]))
    c_n2, c_o2 = 0.8 / (2 * 0.0140067), 0.4 / (2 * 0.015999)
    expected = 2.0 * 7.0e15 * 8000.0 ** -1.6 * np.exp(-113200.0 / 8000.0) * c_n2 * (c_n2 + c_o2)
    assert abs(float(omega[0, 6]) - expected) / expected < 1e-3
    states = GOLDEN["rate_states"][:3]
    for T in GOLDEN["rate_temps"]:
        _, w = mech.net_production_rates(_cuda(states), _cuda(np.full(3, T)))
        w = w.cpu().numpy()
        for row in w:
            m = np.max(np.abs(row))
            assert abs(row.sum()) < (1e-14 * m if m > 1e-10 else 1e-12)


def test_three_species_mechanism():
    """The reference's extensibility case (tests/test_air11_chemistry.py:132-172)."""
    from jax_fluid_sim_b200 import Reaction, ReactionMechanism, Species, make_nasa7
    species = [Species(n, molar_mass=float(w), poly=make_nasa7(200.0, 1000.0, 6000.0, lo, hi))
               for n, w, (lo, hi) in zip(("H2", "O2", "H2O"), GOLDEN["rocket_mw"], GOLDEN["rocket_nasa"])]
    m = ReactionMechanism(species, [Reaction(((0, 2), (1, 1)), ((2, 2),), A=1.0e11, b=0.0, theta=15000.0)])
    states, temps = GOLDEN["rocket_states"], GOLDEN["rocket_temps"]
    rho = _cuda(np.repeat(states, len(temps), axis=0))
    T = _cuda(np.tile(temps, len(states)))
    omega, wdot = m.net_production_rates(rho, T)
    J = m.production_rate_jacobian(rho, T)
    for k in range(len(states) * len(temps)):
        _close(omega[k].cpu(), GOLDEN["rocket_omega"][k], 1e-12)
        _close(wdot[k].cpu(), GOLDEN["rocket_wdot"][k], 1e-12)
        _close(J[k].cpu(), GOLDEN["rocket_jac"][k], 1e-12)
    w = wdot[1].cpu().numpy()          # rich H2/O2 at 2000 K
    assert w[2] > 0 and w[0] < 0 and w[1] < 0 and abs(w.sum()) < 1e-12 * np.max(np.abs(w)) + 1e-12


def _invariants(U, out):
    np.testing.assert_allclose(out[..., 5:].sum(-1), U[..., 0], rtol=1e-12)
    np.testing.assert_array_equal(out[..., :5], U[..., :5])
    assert np.all(out[..., 5:] >= 0.0)


def test_coupler_si_matches_reference():
    """At dt = 1e-7 s the reference's own coupler state does not converge in 16 Newton
    iterations (the iterate oscillates and depends on round-off): invariants only.  At
    dt = 1e-9 s it converges and the species match the reference to 1e-10."""
    from jax_fluid_sim_b200 import ReactingFlowCoupler
    U = GOLDEN["coupler_U"]
    c = ReactingFlowCoupler(max_newton_iters=16)
    out = c.react_block(_cuda(U), float(GOLDEN["coupler_dt"])).cpu().numpy()
    _invariants(U, out)
    assert np.all(out[..., 5 + 7] > 1e-10)
    conv = c.react_block(_cuda(U), float(GOLDEN["coupler_conv_dt"])).cpu().numpy()
    _invariants(U, conv)
    assert np.max(np.abs(conv - GOLDEN["coupler_conv_out"])[..., 5:] / U[..., :1]) < 1e-10


def test_coupler_dimensionless_matches_reference():
    from jax_fluid_sim_b200 import ReactingFlowCoupler
    U, dt = GOLDEN["dimless_U"], float(GOLDEN["dimless_dt"])
    c = ReactingFlowCoupler(max_newton_iters=16, dimensionless=True, reference_temperature=220.0,
                            reference_pressure=500.0, reference_length=0.1)
    out = c.react_block(_cuda(U), dt).cpu().numpy()
    _invariants(U, out)
    assert np.max(np.abs(out - GOLDEN["dimless_out"])[..., 5:] / U[..., :1]) < 2e-5


def _air_block(E, Np, seed):
    """Dimensionless (T_ref 220 K) frozen air between 3000 and 7000 K at Mach 0-8: the
    state a Mach-8 shock layer hands to the coupler."""
    rng = np.random.default_rng(seed)
    U = np.zeros((E, Np, 16))
    rho = 0.5 + 3.0 * rng.random((E, Np))
    vel = 8.0 * np.sqrt(1.4) * rng.random((E, Np))
    T = 3000.0 + 4000.0 * rng.random((E, Np))
    U[..., 0], U[..., 1] = rho, rho * vel
    U[..., 4] = rho * T / 220.0 / 0.4 + 0.5 * rho * vel ** 2
    U[..., 5 + 9], U[..., 5 + 10] = 0.767 * rho, 0.233 * rho
    return U


def test_coupler_matches_oracle_per_element_dt_and_in_place():
    """A sampled block with per-element (local time stepping) dt, updated in place, against
    the oracle node by node (coupling.py:179-197 with an (E,) dt).  The steps are chosen so
    that every node's 12 Newton iterations converge (scaled residual below 5e-12)."""
    from jax_fluid_sim_b200 import ReactingFlowCoupler
    E, Np = 6, 9
    U = _air_block(E, Np, 11)
    dts = 3e-4 * (1.0 + np.arange(E))
    c = ReactingFlowCoupler(dimensionless=True, reference_temperature=220.0, reference_pressure=500.0,
                            reference_length=0.1)
    Ud = _cuda(U)
    out_t = c.react_block(Ud, _cuda(dts), out=Ud)
    assert out_t.data_ptr() == Ud.data_ptr()
    out = Ud.cpu().numpy()
    ref = Coupler(12, True, 220.0, 500.0, 0.1)
    exp = np.stack([ref.react_block(U[e:e + 1], float(dts[e]))[0] for e in range(E)])
    _invariants(U, out)
    assert np.max(np.abs(out - U)[..., 5:]) > 1e-3          # the step does react
    assert np.max(np.abs(out - exp)[..., 5:] / U[..., :1]) < 1e-8


def test_coupler_argument_errors():
    from jax_fluid_sim_b200 import ReactingFlowCoupler
    c = ReactingFlowCoupler()
    with pytest.raises(ValueError, match="expected at least 16"):
        c.react_block(torch.zeros((2, 3, 5), dtype=torch.float64, device="cuda"), 1e-6)
    with pytest.raises(ValueError):
        c.react_block(torch.zeros((2, 3, 16), dtype=torch.float64, device="cuda"), torch.ones(3))
    with pytest.raises(NotImplementedError):
        ReactingFlowCoupler(relaxation=object())
    empty = torch.zeros((0, 27, 16), dtype=torch.float64, device="cuda")
    assert c.react_block(empty, 1e-6).shape == (0, 27, 16)
