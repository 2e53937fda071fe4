"""Ensembles of independent cases in one plan (dgb_plan_set_cases) against the same cases run
alone: three extruded cylinder O-grids of different sizes, Mach numbers and Reynolds numbers,
two checked SSP-RK3 steps with the MOOD limiter at one dt.  Each case inside the ensemble must
equal the case advanced on its own plan (the element and face kernels see the same numbers;
bit-identical is expected, 1e-13 of the field's largest magnitude is required), and the
ensemble's dt is the smallest of the cases' dts.  The single-case path itself is checked
against the oracle on the smallest grid."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MACH = [0.5, 2.0, 3.5]
RE = [200.0, 5.0e3, 1.0e5]
GRIDS = [(16, 6, 15.0), (24, 8, 10.0), (20, 5, 12.0)]


def _cases():
    from jax_fluid_sim_b200 import meshgen
    sources = [meshgen.cylinder_o_grid(nt, nr, outer_radius=ro) for nt, nr, ro in GRIDS]
    far = [np.array([1.0, m * np.sqrt(1.4), 0.0, 0.0, 1.0]) for m in MACH]
    mu = [f[1] / re for f, re in zip(far, RE)]
    return sources, far, mu


def _integrator(jfs, op, graph=False):
    lim = jfs.HybridMOODSubcellLimiter(op, positivity=jfs.HybridPositivityLimiter(op))
    return jfs.HybridSSPRK3(op, cfl=0.3, limiter=lim, graph=graph)


@pytest.mark.parametrize("degree", [2, 3])
def test_ensemble_equals_cases_alone(degree):
    import jax_fluid_sim_b200 as jfs
    from jax_fluid_sim_b200.ensemble import HybridEnsemble
    sources, far, mu = _cases()
    ens = HybridEnsemble(sources, far, mu, polynomial_degree=degree)
    U = ens.freestream_states()
    integ = _integrator(jfs, ens.operator, graph=True)
    dt = integ.stable_dt(U, ens.boundary)
    alone, dts = [], []
    for c, src in enumerate(sources):
        solver = jfs.HybridCompressibleSolver(jfs.HybridMesh(src), polynomial_degree=degree, dynamic_viscosity=mu[c])
        op = jfs.HybridNavierStokesOperator(solver)
        bc = jfs.FarfieldWallBoundary(solver, far[c])
        Uc = solver.uniform_state_blocks(far[c][0], far[c][1:4], far[c][4])
        it = _integrator(jfs, op)
        dts.append(it.stable_dt(Uc, bc))
        alone.append((it, Uc, bc))
    assert dt == pytest.approx(min(dts), rel=1e-15)
    for _ in range(2):
        assert bool(integ.checked_step_inplace(U, dt, ens.boundary).view(torch.int32)[0].item())
        for it, Uc, bc in alone:
            it.checked_step_inplace(Uc, dt, bc)
    for c, part in enumerate(ens.split(U)):
        Uc = alone[c][1]
        for k in part:
            scale = Uc[k].abs().amax(dim=(0, 1))
            err = ((part[k] - Uc[k]).abs().amax(dim=(0, 1)) / scale).max().item()
            assert err <= 1e-13, (c, k, err)


def test_cylinder_grid_against_oracle():
    """The cylinder O-grid's residual (isothermal no-slip wall, far field, symmetry planes) at
    P2 against the oracle, from a perturbed Mach-2 state."""
    import jax_fluid_sim_b200 as jfs
    from oracle.dg import Operator
    from oracle.mesh import Mesh, MeshSource
    from oracle.physics import FarfieldWallBoundary, Gas
    sources, far, mu = _cases()
    src, f, m = sources[1], far[1], mu[1]
    solver = jfs.HybridCompressibleSolver(jfs.HybridMesh(src), polynomial_degree=2, dynamic_viscosity=m)
    op = jfs.HybridNavierStokesOperator(solver)
    bc = jfs.FarfieldWallBoundary(solver, f, wall_temperature=1.2)

    def prim(x):
        W = np.broadcast_to(f, x.shape[:-1] + (5,)).copy()
        W[..., 0] *= 1.0 + 0.1 * np.sin(x[..., 0]) * np.cos(0.5 * x[..., 1])
        W[..., 2] = 0.2 * np.cos(x[..., 0])
        return W

    states = solver.state_blocks_from_primitive_function(op, prim)
    mesh = Mesh(MeshSource(src.points, src.cells, src.physical, src.field_data))
    gas = Gas(dynamic_viscosity=m)
    oop = Operator(mesh, gas, 2)
    obc = FarfieldWallBoundary(gas, mesh.physical_names, f, wall_temperature=1.2)
    U = {k: v.cpu().numpy() for k, v in states.items()}
    inv, vis = op.inviscid_rhs(states, bc), op.viscous_rhs(states, bc)
    rinv, rvis = oop.inviscid_rhs(U, obc), oop.viscous_rhs(U, obc)
    for k in U:
        for got, ref in ((inv[k], rinv[k]), (vis[k], rvis[k])):
            scale = max(np.abs(ref).max(), 1e-300)
            assert np.abs(got.cpu().numpy() - ref).max() <= 1e-9 * scale
