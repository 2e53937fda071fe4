"""The reacting configuration (Mach-8 sphere, 11 Air-11 species carried as conserved variables,
isothermal wall) on the smallest O/H grid at P2 against the oracle: one checked SSP-RK3 step
with the MOOD limiter, then the operator-split chemistry source with the dimensionless coupler
(T_ref 220 K, p_ref 500 Pa, L_ref 0.2 m) on the hottest elements.

Tolerance: the step to 1e-9 of each field's largest magnitude (float64, different summation
order); the reacted species to 1e-5 of the node density (the Newton matrix I - dt J is stiff
here, as in the coupler fixture test); the species densities sum to the mixture density as
closely as the oracle's after the step (the CWENO-Z subcell reconstruction is per species) and to
1e-12 relative after the source, which renormalises them."""

import numpy as np
import pytest
import torch

from jax_fluid_sim_b200 import workloads

pytestmark = pytest.mark.gpu


def test_reacting_step_against_oracle():
    import jax_fluid_sim_b200 as jfs
    from oracle.chemistry import Coupler
    from oracle.dg import Operator, PositivityLimiter, TimeIntegrator
    from oracle.mesh import Mesh, MeshSource
    from oracle.physics import FarfieldWallBoundary, Gas
    from oracle.subcell import MOODLimiter
    solver, op, bc, coupler, states = workloads.reacting_case("tiny", degree=2)
    src = workloads.reacting_mesh("tiny")
    mesh = Mesh(MeshSource(src.points, src.cells, src.physical, src.field_data))
    gas = Gas(dynamic_viscosity=solver.dynamic_viscosity, n_species=11)
    oop = Operator(mesh, gas, 2)
    far = workloads.reacting_farfield()
    obc = FarfieldWallBoundary(gas, mesh.physical_names, far, wall_temperature=300.0 / 220.0)
    U = {k: v.cpu().numpy() for k, v in states.items()}
    oint = TimeIntegrator(oop, cfl=0.3, limiter=MOODLimiter(oop, positivity=PositivityLimiter(oop)))
    dt = oint.stable_dt(U)
    ref, ref_valid, _, _ = oint.checked_step(U, dt, obc)
    lim = jfs.HybridMOODSubcellLimiter(op, positivity=jfs.HybridPositivityLimiter(op))
    got, valid, _, _ = jfs.HybridSSPRK3(op, cfl=0.3, limiter=lim).checked_step(states, dt, bc)
    assert valid == ref_valid
    for k in ref:
        scale = np.maximum(np.abs(ref[k]).max(axis=(0, 1)), 1e-300)
        err = np.abs(got[k].cpu().numpy() - ref[k]).max(axis=(0, 1)) / scale
        assert err.max() <= 1e-9, err
    # the subcell scheme reconstructs every species with its own CWENO-Z weights, so the sum of
    # the species densities drifts from the mixture density by the weights' nonlinearity; the
    # drift must match the oracle's, and the coupler's renormalisation removes it
    drift = max(float(np.max(np.abs(ref[k][..., 5:].sum(-1) - ref[k][..., 0]) / ref[k][..., 0])) for k in ref)
    assert drift < 1e-6
    assert workloads.species_closure(got) <= 2.0 * drift + 1e-13
    oc = Coupler(16, True, 220.0, 500.0, 0.2)
    for k in ref:
        reacted = coupler.react_block(got[k], dt).cpu().numpy()
        np.testing.assert_array_equal(reacted[..., :5], got[k].cpu().numpy()[..., :5])
        assert workloads.species_closure({k: torch.as_tensor(reacted)}) <= 1e-12
        # the oracle coupler is a per-node Python loop: compare the 8 hottest elements
        hot = np.argsort(-(ref[k][..., 4] / ref[k][..., 0]).max(axis=1))[:8]
        oref = oc.react_block(ref[k][hot], dt)
        assert np.max(np.abs(reacted[hot][..., 5:] - oref[..., 5:]) / ref[k][hot][..., :1]) <= 1e-5


def test_reacting_steps_and_shock_position_against_oracle():
    """Twenty steps of the reacting sphere (each a checked MOOD step, then the Air-11 source on every
    node) on the smallest grid from the shocked start, against the oracle's own run
    (tests/golden/make_golden_reacting.py, the batched oracle coupler): the same admissibility in
    every step, the bow shock's position on the stagnation line after every step (it forms at the
    wall and stands off to x = -0.804 within these steps) to 1e-10, and the final state at 2,048
    seeded nodes: the flow to 1e-10 of each field's largest magnitude, the species to 1e-9 of the
    node density (measured: 2e-14 and 2e-13)."""
    from pathlib import Path
    import jax_fluid_sim_b200 as jfs
    G = np.load(Path(__file__).resolve().parent / "golden" / "reacting_tiny.npz")
    solver, op, bc, coupler, U = workloads.reacting_case("tiny", degree=2)
    integ = jfs.HybridSSPRK3(op, cfl=0.3, limiter=jfs.HybridMOODSubcellLimiter(
        op, positivity=jfs.HybridPositivityLimiter(op)))
    dt = float(G["dt"])
    assert abs(integ.stable_dt(U, bc) - dt) <= 1e-12 * dt
    xyz = op.solution_node_coordinates["hexahedron"]
    shock, valid = [workloads.stagnation_shock_x(xyz, U["hexahedron"][..., 0].cpu().numpy())], []
    for _ in range(int(G["steps"])):
        U, ok, _, _ = integ.checked_step(U, dt, bc)
        valid.append(bool(ok))
        U = {k: coupler.react_block(v, dt) for k, v in U.items()}
        shock.append(workloads.stagnation_shock_x(xyz, U["hexahedron"][..., 0].cpu().numpy()))
    assert valid == list(G["valid"])
    np.testing.assert_allclose(shock, G["shock_x"], rtol=0, atol=1e-10, equal_nan=True)
    assert np.isnan(shock[0]) and shock[-1] < -0.8
    got = U["hexahedron"].reshape(-1, U["hexahedron"].shape[-1]).cpu().numpy()[G["sample_index"]]
    ref = G["sample_state"]
    flow = (np.abs(got - ref)[:, :5].max(axis=0) / np.abs(ref[:, :5]).max(axis=0)).max()
    assert flow <= 1e-10, flow
    species = np.max(np.abs(got - ref)[:, 5:] / ref[:, :1])
    assert species <= 1e-9, species
