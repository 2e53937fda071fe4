"""MOOD subcell tables built on the device (dgb_plan_build_subcells, dgb_plan_match_subcell_faces)
against the host construction (numpy projection and least-squares inverse, the native subface
metrics, host subface matching; hybrid/subcell.py:277-396,473-533).

With every element troubled, the subcell recompute reads every table: projections,
reconstructions, volumes, centres, subface normals and areas, the matched neighbour subfaces.
Both plans must then give the same state to 1e-11 of each field's largest magnitude (the device
sums the projections and the Gram matrices in a different order than numpy's matrix products);
the subcell reconstructions TVD and CWENO-Z read the centres as well.
"""

import numpy as np
import pytest
import torch

from .conftest import GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu


def _operators(source, degree, mu, species=()):
    from jax_fluid_sim_b200 import HybridCompressibleSolver, HybridMesh, HybridNavierStokesOperator
    solver = HybridCompressibleSolver(HybridMesh(source), polynomial_degree=degree, dynamic_viscosity=mu,
                                      species_names=species)
    dev = HybridNavierStokesOperator(solver)
    host = HybridNavierStokesOperator(solver)
    return solver, dev, host


@pytest.mark.parametrize("case", GOLDEN_CASES + ["sphere"])
@pytest.mark.parametrize("reconstruction", ["constant", "tvd", "weno"])
def test_device_subcell_tables_match_host(case, reconstruction):
    from jax_fluid_sim_b200 import HybridSubcellFV
    from jax_fluid_sim_b200 import workloads
    if case == "sphere":
        solver, dev, host = _operators(workloads.sphere_mesh("tiny"), 3, 1e-3)
        states = workloads.sphere_shock_state(solver, dev, 3.0 * 1.4 ** 0.5)
    else:
        g = load_golden(case)
        solver, dev, host = _operators(g["source"], int(g["degree"]), float(g["mu"]),
                                       tuple(str(n) for n in g.get("species", ())))
        states = {k: torch.as_tensor(g[f"U_shocked_{k}"], device="cuda") for k in g["block_names"]}
    dev.native.enable_mood("reference", tables="device")
    host.native.enable_mood("reference", tables="host")
    flags = {k: torch.ones(v.shape[0], dtype=torch.bool, device="cuda") for k, v in states.items()}
    rhs = dev.inviscid_rhs(states)
    cand = {k: states[k] + 1e-3 * rhs[k] for k in states}
    outs = []
    for op in (dev, host):
        fv = HybridSubcellFV(op, reconstruction=reconstruction)
        outs.append(fv.recompute(states, cand, 1e-3, flags))
    for k in states:
        a, b = outs[0][k].cpu().numpy(), outs[1][k].cpu().numpy()
        scale = np.maximum(np.abs(b).max(axis=(0, 1)), 1e-300)
        err = (np.abs(a - b).max(axis=(0, 1)) / scale).max()
        assert err <= 1e-11, (k, err)
