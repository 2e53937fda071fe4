"""dgb_ssprk3_step_graph (the checked step replayed from a CUDA graph) against dgb_ssprk3_step.

The graph holds the same kernels in the same order, so the states must be bit-identical:
on the first call (capture), on a replay, after dt changes (a new capture) and after a
parameter change of the plan."""

import numpy as np
import pytest
import torch

from .test_gpu_parity import setup

pytestmark = pytest.mark.gpu


def _integrators(op, mood, graph):
    from jax_fluid_sim_b200 import HybridMOODSubcellLimiter, HybridPositivityLimiter, HybridSSPRK3
    pos = HybridPositivityLimiter(op)
    lim = HybridMOODSubcellLimiter(op, positivity=pos) if mood else pos
    return HybridSSPRK3(op, cfl=0.3, limiter=lim, graph=graph)


@pytest.mark.parametrize("case,mood", [("box_p3", True), ("mixed_p2", True), ("box_p2", False)])
def test_graph_step_is_bit_identical(case, mood):
    g, solver, op, bc = setup(case)
    states = {k: g[f"U_shocked_{k}"] for k in g["block_names"]}
    direct, graphed = _integrators(op, mood, False), _integrators(op, mood, True)
    dt = direct.stable_dt(states, bc)
    Ud = op.to_device({k: np.array(v, copy=True) for k, v in states.items()})
    Ug = op.to_device({k: np.array(v, copy=True) for k, v in states.items()})
    for k_dt in (dt, dt, 0.5 * dt, 0.5 * dt):
        direct.checked_step_inplace(Ud, k_dt, bc)
        sd = direct._status_tuple()
        graphed.checked_step_inplace(Ug, k_dt, bc)
        sg = graphed._status_tuple()
        for k in Ud:
            assert torch.equal(Ud[k], Ug[k])
        assert sd[0] == sg[0] and (sd[1] == sg[1] or np.isnan(sd[1]))
    # a parameter change (far-field) must not replay the stale graph
    from jax_fluid_sim_b200 import FarfieldWallBoundary
    bc2 = FarfieldWallBoundary(solver, np.asarray(g["farfield"]) * np.array([1.1, 1.0, 1.0, 1.0, 1.2]),
                               wall_temperature=None if np.isnan(float(g["wall_temperature"])) else float(g["wall_temperature"]))
    direct.checked_step_inplace(Ud, dt, bc2)
    graphed.checked_step_inplace(Ug, dt, bc2)
    for k in Ud:
        assert torch.equal(Ud[k], Ug[k])
