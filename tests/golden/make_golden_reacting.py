"""Fixture of the reacting sphere over several steps, made by the oracle (CPU, float64).

The smallest O/H sphere grid at P2 with the 11 Air-11 species (Mach 8, Re_D 2.6e5, isothermal
wall 300 K / 220 K), from the shocked start: STEPS steps at the start's stable dt, each a checked
SSP-RK3 step with the MOOD limiter followed by the dimensionless Air-11 coupler on every node
(run_hybrid_sphere.py:292-312).  Stored: dt, the admissibility of every step, the shock position
on the stagnation line after every step, and the final state at a seeded sample of nodes.

    python tests/golden/make_golden_reacting.py        # writes tests/golden/reacting_tiny.npz
"""

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

STEPS = 20
SAMPLE = 2048


def main():
    from jax_fluid_sim_b200 import workloads
    from jax_fluid_sim_b200.air11 import AIR11_SPECIES
    from jax_fluid_sim_b200.mesh import HybridMesh
    from jax_fluid_sim_b200.plan import Plan
    from jax_fluid_sim_b200.solver import HybridCompressibleSolver
    from oracle.chemistry import Coupler, batch_react_block
    from oracle.dg import Operator, PositivityLimiter, TimeIntegrator
    from oracle.mesh import Mesh, MeshSource
    from oracle.physics import FarfieldWallBoundary, Gas
    from oracle.subcell import MOODLimiter

    src = workloads.reacting_mesh("tiny")
    hmesh = HybridMesh(src)
    plan = Plan(hmesh, 2)
    far = workloads.reacting_farfield()
    mu = far[1] / 2.6e5
    # the start state at the solution nodes (the same nodes and layout as the oracle's)
    solver = HybridCompressibleSolver(hmesh, species_names=tuple(s.name for s in AIR11_SPECIES), gamma=1.4,
                                      polynomial_degree=2, dynamic_viscosity=mu)
    U = {bp.etype: solver.primitive_to_conserved(workloads.reacting_start(bp.node_xyz)) for bp in plan.blocks}
    xyz = plan.blocks[0].node_xyz
    mesh = Mesh(MeshSource(src.points, src.cells, src.physical, src.field_data))
    gas = Gas(dynamic_viscosity=mu, n_species=11)
    op = Operator(mesh, gas, 2)
    bc = FarfieldWallBoundary(gas, mesh.physical_names, far, wall_temperature=300.0 / 220.0)
    integ = TimeIntegrator(op, cfl=0.3, limiter=MOODLimiter(op, positivity=PositivityLimiter(op)))
    coupler = Coupler(12, True, 220.0, 500.0, 0.2)
    dt = integ.stable_dt(U)
    valid, shock = [], [workloads.stagnation_shock_x(xyz, U["hexahedron"][..., 0])]
    for step in range(STEPS):
        t = time.time()
        U, ok, _, _ = integ.checked_step(U, dt, bc)
        U = {k: batch_react_block(coupler, v, dt) for k, v in U.items()}
        valid.append(bool(ok))
        shock.append(workloads.stagnation_shock_x(xyz, U["hexahedron"][..., 0]))
        print(f"step {step + 1}: valid {ok} shock x {shock[-1]:.12f} ({time.time() - t:.1f} s)", flush=True)
    final = U["hexahedron"].reshape(-1, U["hexahedron"].shape[-1])
    idx = np.sort(np.random.default_rng(0).choice(len(final), size=SAMPLE, replace=False))
    np.savez(Path(__file__).resolve().parent / "reacting_tiny.npz", dt=dt, steps=STEPS, valid=np.array(valid),
             shock_x=np.array(shock), sample_index=idx, sample_state=final[idx])


if __name__ == "__main__":
    main()
