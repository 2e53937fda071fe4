"""The benchmark's sphere grid (smallest O/H grid, 416 P3 hexahedra, about half of them affine)
on the GPU against the oracle: residuals of a smooth state, one checked MOOD step from the
benchmark's shocked start, and the affine fast path against the dense metrics.

Tolerance: 1e-9 of each field's largest magnitude against the oracle (float64, different
summation order); the affine path matches the dense one to 1e-12 (its tensor-product inverse
mass matrix equals the quadrature one to round-off)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GAMMA, MACH, RE, T_RATIO = 1.4, 3.0, 1.0e5, 300.0 / 220.0


def _close(a, b, tol):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    scale = max(np.max(np.abs(b)), 1e-300)
    err = np.max(np.abs(a - b)) / scale
    assert err <= tol, f"relative error {err:.3e} > {tol:.1e}"


@pytest.fixture(scope="module")
def sphere():
    import jax_fluid_sim_b200 as jfs
    from jax_fluid_sim_b200 import meshgen
    from oracle.mesh import Mesh, MeshSource
    from oracle.physics import FarfieldWallBoundary, Gas
    src = meshgen.sphere_oh_grid(n=4, n_radial=2, outer=((1, 3), (1, 1), (1, 1)))
    u = MACH * np.sqrt(GAMMA)
    mu = u / RE
    farfield = np.array([1.0, u, 0.0, 0.0, 1.0])
    solver = jfs.HybridCompressibleSolver(jfs.HybridMesh(src), polynomial_degree=3, dynamic_viscosity=mu)
    op = jfs.HybridNavierStokesOperator(solver)
    dense = jfs.HybridNavierStokesOperator(solver, affine=False)
    bc = jfs.FarfieldWallBoundary(solver, farfield, wall_temperature=T_RATIO)
    mesh = Mesh(MeshSource(src.points, src.cells, src.physical, src.field_data))
    gas = Gas(dynamic_viscosity=mu)
    from oracle.dg import Operator
    oop = Operator(mesh, gas, 3)
    obc = FarfieldWallBoundary(gas, mesh.physical_names, farfield, wall_temperature=T_RATIO)
    return dict(jfs=jfs, op=op, dense=dense, bc=bc, oop=oop, obc=obc, gas=gas, mesh=mesh, u=u, solver=solver)


def _node_xyz(mesh, block):
    from oracle.elements import RefElement
    nodes = RefElement(block.element_type, 3).nodes
    return np.einsum("qi,eid->eqd", RefElement(block.element_type, 1).basis(nodes), mesh.points[block.connectivity])


def test_affine_fraction(sphere):
    assert 0.3 < sphere["op"].native.affine_fraction < 0.9


def test_smooth_residuals_against_oracle(sphere):
    gas, mesh, u = sphere["gas"], sphere["mesh"], sphere["u"]
    states = {}
    for b in mesh.element_blocks:
        x = _node_xyz(mesh, b)
        W = np.zeros(x.shape[:-1] + (5,))
        W[..., 0] = 1.0 + 0.2 * np.sin(1.3 * x[..., 0]) * np.cos(0.7 * x[..., 1])
        W[..., 1] = u * (1.0 + 0.1 * np.cos(x[..., 2]))
        W[..., 2] = 0.3 * np.sin(x[..., 0] + x[..., 2])
        W[..., 3] = -0.2 * np.cos(x[..., 1])
        W[..., 4] = 1.0 + 0.3 * np.cos(0.9 * x[..., 0] - 0.4 * x[..., 2])
        states[b.element_type] = gas.to_conserved(W)
    oop, obc = sphere["oop"], sphere["obc"]
    ref_inv = oop.inviscid_rhs(states, obc)
    ref_vis = oop.viscous_rhs(states, obc)
    for op in (sphere["op"], sphere["dense"]):
        inv, vis = op.inviscid_rhs(states, sphere["bc"]), op.viscous_rhs(states, sphere["bc"])
        for k in states:
            _close(inv[k], ref_inv[k], 1e-9)
            _close(vis[k], ref_vis[k], 1e-9)
    a_inv = sphere["op"].inviscid_rhs(states, sphere["bc"])
    d_inv = sphere["dense"].inviscid_rhs(states, sphere["bc"])
    a_vis = sphere["op"].viscous_rhs(states, sphere["bc"])
    d_vis = sphere["dense"].viscous_rhs(states, sphere["bc"])
    for k in states:
        _close(a_inv[k], d_inv[k].cpu().numpy(), 1e-12)
        _close(a_vis[k], d_vis[k].cpu().numpy(), 1e-12)


def test_shocked_mood_step_against_oracle(sphere):
    """The benchmark's start: the Mach-3 normal-shock state in the elements whose centroid is
    inside r < 0.65, the free stream elsewhere; one checked SSP-RK3 step with MOOD (CWENO-Z)."""
    jfs, gas, mesh, u = sphere["jfs"], sphere["gas"], sphere["mesh"], sphere["u"]
    from oracle.dg import PositivityLimiter, TimeIntegrator
    from oracle.subcell import MOODLimiter
    g, M = GAMMA, MACH
    rho2 = (g + 1) * M ** 2 / ((g - 1) * M ** 2 + 2)
    p2 = 1 + 2 * g / (g + 1) * (M ** 2 - 1)
    states = {}
    for b in mesh.element_blocks:
        x = _node_xyz(mesh, b)
        inside = np.broadcast_to(np.linalg.norm(x.mean(axis=1), axis=-1)[:, None] < 0.65, x.shape[:-1])
        W = np.zeros(x.shape[:-1] + (5,))
        W[..., 0] = np.where(inside, rho2, 1.0)
        W[..., 1] = np.where(inside, u / rho2, u)
        W[..., 4] = np.where(inside, p2, 1.0)
        states[b.element_type] = gas.to_conserved(W)
    oop = sphere["oop"]
    integ = TimeIntegrator(oop, cfl=0.3, limiter=MOODLimiter(oop, positivity=PositivityLimiter(oop)))
    dt = integ.stable_dt(states)
    ref, ref_valid, ref_rmin, ref_pmin = integ.checked_step(states, dt, sphere["obc"])
    op = sphere["op"]
    gi = jfs.HybridSSPRK3(op, cfl=0.3, limiter=jfs.HybridMOODSubcellLimiter(op, positivity=jfs.HybridPositivityLimiter(op)))
    got, valid, rmin, pmin = gi.checked_step(states, dt, sphere["bc"])
    assert valid == ref_valid
    assert rmin == pytest.approx(ref_rmin, rel=1e-9) and pmin == pytest.approx(ref_pmin, rel=1e-9)
    for k in ref:
        _close(got[k], ref[k], 1e-9)


def test_shocked_mood_flags_bit_exact(sphere):
    """The MOOD troubled-cell flags on the benchmark's grid bit for bit against the oracle
    (hybrid/limiter.py:285-300): on the shocked start and on the first stage's DG candidate
    U + dt R(U), the state the detector judges inside the checked step."""
    jfs, gas, mesh, u = sphere["jfs"], sphere["gas"], sphere["mesh"], sphere["u"]
    from oracle.dg import PositivityLimiter, TimeIntegrator, TroubledCellSensor, mood_troubled
    g, M = GAMMA, MACH
    rho2 = (g + 1) * M ** 2 / ((g - 1) * M ** 2 + 2)
    p2 = 1 + 2 * g / (g + 1) * (M ** 2 - 1)
    states = {}
    for b in mesh.element_blocks:
        x = _node_xyz(mesh, b)
        inside = np.broadcast_to(np.linalg.norm(x.mean(axis=1), axis=-1)[:, None] < 0.65, x.shape[:-1])
        W = np.zeros(x.shape[:-1] + (5,))
        W[..., 0] = np.where(inside, rho2, 1.0)
        W[..., 1] = np.where(inside, u / rho2, u)
        W[..., 4] = np.where(inside, p2, 1.0)
        states[b.element_type] = gas.to_conserved(W)
    oop, obc = sphere["oop"], sphere["obc"]
    opos = PositivityLimiter(oop)
    dt = TimeIntegrator(oop, cfl=0.3, limiter=opos).stable_dt(states)
    rhs = oop.rhs(states, obc)
    candidate = {k: states[k] + dt * rhs[k] for k in states}
    op = sphere["op"]
    lim = jfs.HybridMOODSubcellLimiter(op, positivity=jfs.HybridPositivityLimiter(op))
    seen = 0
    for s in (states, candidate):
        ref = mood_troubled(oop, opos, TroubledCellSensor(oop), s)
        got = lim.troubled(s)
        for k in ref:
            np.testing.assert_array_equal(got[k].cpu().numpy(), ref[k])
            seen += int(ref[k].sum())
    assert seen > 0, "the shocked start should flag some elements"
