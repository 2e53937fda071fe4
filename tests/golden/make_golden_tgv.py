"""Golden fixture of the Taylor-Green vortex configuration, made by the CPU oracle.

    python tests/golden/make_golden_tgv.py

Periodic [0, 2 pi]^3 of 16^3 hexahedra at P2, gamma 1.4, Pr 0.71, Re 1600, Mach 0.1; ten
checked SSP-RK3 steps at CFL 0.3, dt from the oracle's stable_dt before each step (HLLC + BR2,
no limiter).  The full state is 4096 x 27 x 5 values, so the fixture keeps the dt sequence,
the conserved totals, each field's largest magnitude and the values at 4096 seeded
(element, node) samples of the initial inviscid and viscous residuals and of the final state.
Takes about five minutes on one core.
"""

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from jax_fluid_sim_b200 import workloads  # noqa: E402  (numpy mesh and initial state only)
from oracle.dg import Operator, TimeIntegrator  # noqa: E402
from oracle.elements import RefElement  # noqa: E402
from oracle.mesh import Mesh, MeshSource  # noqa: E402
from oracle.physics import Gas  # noqa: E402

N, DEGREE, STEPS, CFL = 16, 2, 10, 0.3


def totals(geo, U):
    el = geo.element[0]
    B = RefElement("hexahedron", DEGREE).B
    return np.einsum("eq,qn,env->v", el.wdet, B, U)


def main():
    src = workloads.tgv_mesh(N)
    mesh = Mesh(MeshSource(src.points, src.cells, src.physical, src.field_data, src.periodic_map))
    gas = Gas(dynamic_viscosity=1.0 / 1600.0, prandtl=0.71)
    op = Operator(mesh, gas, DEGREE)
    block = mesh.element_blocks[0]
    ref = RefElement(block.element_type, DEGREE)
    x = np.einsum("qi,eid->eqd", RefElement(block.element_type, 1).basis(ref.nodes), mesh.points[block.connectivity])
    U0 = gas.to_conserved(workloads.tgv_primitive(x))
    states = {block.element_type: U0}
    rng = np.random.default_rng(0)
    elem = rng.integers(0, U0.shape[0], 4096)
    node = rng.integers(0, U0.shape[1], 4096)
    inv = op.inviscid_rhs(states)[block.element_type]
    vis = op.viscous_rhs(states)[block.element_type]
    integ = TimeIntegrator(op, cfl=CFL)
    dts = []
    for s in range(STEPS):
        dt = integ.stable_dt(states)
        states, valid, _, _ = integ.checked_step(states, dt)
        assert valid
        dts.append(dt)
        print("step", s, dt, flush=True)
    U = states[block.element_type]
    np.savez_compressed(HERE / "tgv_p2_16.npz", elem=elem, node=node, dt=np.array(dts),
                        rhs_inviscid=inv[elem, node], rhs_viscous=vis[elem, node],
                        rhs_inviscid_scale=np.abs(inv).max(axis=(0, 1)), rhs_viscous_scale=np.abs(vis).max(axis=(0, 1)),
                        final=U[elem, node], final_scale=np.abs(U).max(axis=(0, 1)),
                        totals0=totals(op.geo, U0), totals=totals(op.geo, U))


if __name__ == "__main__":
    main()
