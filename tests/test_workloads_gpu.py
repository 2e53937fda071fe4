"""The Taylor-Green and isentropic-vortex workloads on the GPU against the oracle: residuals and
checked SSP-RK3 steps on small periodic boxes (hexahedra for Taylor-Green; the conforming
hexahedron/prism/tetrahedron box for the vortex at P1-P3), and conservation of mass, momentum
and energy to round-off on the periodic boxes.

Tolerance: 1e-9 of each field's largest magnitude against the oracle (float64, different
summation order); 5e-5 for precision='mixed' residuals on this box (float32 sums over up to 125
volume points per node; observed 2.1e-5 at P3); totals conserved to 1e-13 relative."""

import numpy as np
import pytest
import torch

from jax_fluid_sim_b200 import HybridSSPRK3, workloads

pytestmark = pytest.mark.gpu


def _close(a, b, tol):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    scale = max(np.max(np.abs(b)), 1e-300)
    err = np.max(np.abs(a - b)) / scale
    assert err <= tol, f"relative error {err:.3e} > {tol:.1e}"


def _oracle_operator(source, degree, **gas):
    from oracle.dg import Operator
    from oracle.mesh import Mesh, MeshSource
    from oracle.physics import Gas
    mesh = Mesh(MeshSource(source.points, source.cells, source.physical, source.field_data, source.periodic_map))
    return Operator(mesh, Gas(**gas), degree)


def _totals(op, states):
    out = np.zeros(5)
    for name, bp in zip(op.names, op.plan.blocks):
        U = states[name].detach().cpu().numpy() if isinstance(states[name], torch.Tensor) else states[name]
        out += np.einsum("eq,qn,env->v", bp.wdet, bp.ref.B, U)
    return out


def _host(states):
    return {k: v.detach().cpu().numpy() for k, v in states.items()}


def test_taylor_green_against_oracle():
    """4^3 periodic hexahedra at P2, Re 1600, Pr 0.71, Mach 0.1: residuals and three steps."""
    from oracle.dg import TimeIntegrator
    solver, op, states = workloads.tgv_case(n=4, degree=2)
    oop = _oracle_operator(workloads.tgv_mesh(4), 2, dynamic_viscosity=1 / 1600, prandtl=0.71)
    U = _host(states)
    ref_inv, ref_vis = oop.inviscid_rhs(U), oop.viscous_rhs(U)
    inv, vis = op.inviscid_rhs(states), op.viscous_rhs(states)
    for k in U:
        _close(inv[k], ref_inv[k], 1e-9)
        _close(vis[k], ref_vis[k], 1e-9)
    oint = TimeIntegrator(oop, cfl=0.3)
    integ = HybridSSPRK3(op, cfl=0.3)
    dt = oint.stable_dt(U)
    assert integ.stable_dt(states) == pytest.approx(dt, rel=1e-12)
    ref, cur = U, {k: v.clone() for k, v in states.items()}
    for _ in range(3):
        ref = oint.checked_step(ref, dt)[0]
        status = integ.checked_step_inplace(cur, dt)
    assert bool(status.view(torch.int32)[0].item())
    for k in U:
        _close(cur[k], ref[k], 1e-9)
    t0, t1 = _totals(op, U), _totals(op, cur)
    assert np.all(np.abs(t1 - t0) <= 1e-13 * np.maximum(np.abs(t0), np.abs(t0).max()))


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_vortex_on_hybrid_box_against_oracle(degree):
    """(4, 3, 4) cubes of hexahedra, prism pairs and Kuhn tetrahedra, jittered 10 %: the Euler
    residual (affine fast path and per-element tables, float64 and mixed) and one checked step."""
    from jax_fluid_sim_b200 import meshgen
    from oracle.dg import TimeIntegrator
    from jax_fluid_sim_b200.mesh import HybridMesh
    from jax_fluid_sim_b200 import HybridCompressibleSolver, HybridEulerOperator
    src = meshgen.hybrid_box((4, 3, 4), jitter=0.1, seed=1)
    solver = HybridCompressibleSolver(HybridMesh(src), polynomial_degree=degree)
    op = HybridEulerOperator(solver)
    # a wider vortex so that P1-P3 on this coarse box see it
    states = solver.state_blocks_from_primitive_function(op, lambda x: workloads.vortex_primitive(x, radius=0.2))
    oop = _oracle_operator(src, degree)
    U = _host(states)
    ref = oop.inviscid_rhs(U)
    got = op.rhs(states)
    tuned = HybridEulerOperator(solver)
    widths = tuned.autotune(states)
    assert set(widths) == {"traces", "volume", "finalize"}
    assert all(w in (16, 32, 64, 128) for row in widths.values() for w in row.values())
    after = tuned.rhs(states)
    mixed = op.with_precision("mixed").rhs(states)
    dense = HybridEulerOperator(solver, affine=False).rhs(states)
    for k in U:
        _close(got[k], ref[k], 1e-9)
        _close(after[k], got[k].cpu().numpy(), 1e-12)
        _close(dense[k], ref[k], 1e-9)
        _close(mixed[k], ref[k], 5e-5)
    oint = TimeIntegrator(oop, cfl=0.3)
    dt = oint.stable_dt(U)
    res, valid, _, _ = HybridSSPRK3(op, cfl=0.3).checked_step(states, dt)
    ref_step = oint.checked_step(U, dt)[0]
    assert valid
    for k in U:
        _close(res[k], ref_step[k], 1e-9)
    t0, t1 = _totals(op, U), _totals(op, res)
    assert np.all(np.abs(t1 - t0) <= 1e-13 * np.abs(t0).max())


def test_vortex_short_run_error_decreases_with_degree():
    """A tenth of a period on the 6^3 box: the density L2 error against the exact vortex falls
    with the degree (each degree at least 2x better), and every step stays admissible."""
    errors = []
    for degree in (1, 2, 3):
        solver, op, states = workloads.vortex_case(n=6, degree=degree, radius=0.15)
        integ = HybridSSPRK3(op, cfl=0.3)
        t = 0.1 * workloads.vortex_period()
        steps, dt = workloads.equal_steps(t, workloads.convective_dt(op, states, 0.3))
        assert workloads.advance(integ, states, steps, dt) and steps > 0
        errors.append(workloads.l2_density_error(op, states, lambda x: workloads.vortex_primitive(x, t, radius=0.15)))
    assert errors[1] < 0.5 * errors[0] and errors[2] < 0.5 * errors[1], errors


def test_taylor_green_full_config_against_golden():
    """The Taylor-Green configuration itself (16^3 hexahedra, P2, ten steps at CFL 0.3) against
    the oracle's run stored in tests/golden/tgv_p2_16.npz (make_golden_tgv.py): initial
    residuals and the final state at 4096 seeded nodes, the dt sequence, and conservation."""
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / "tgv_p2_16.npz")
    solver, op, states = workloads.tgv_case(n=16, degree=2)
    elem, node = torch.as_tensor(g["elem"], device="cuda"), torch.as_tensor(g["node"], device="cuda")
    inv, vis = op.inviscid_rhs(states)["hexahedron"], op.viscous_rhs(states)["hexahedron"]
    for got, key in ((inv, "rhs_inviscid"), (vis, "rhs_viscous")):
        err = np.abs(got[elem, node].cpu().numpy() - g[key]) / np.where(g[f"{key}_scale"] > 0, g[f"{key}_scale"], 1.0)
        assert err.max() <= 1e-9, (key, err.max())
    integ = HybridSSPRK3(op, cfl=0.3)
    t0 = _totals(op, states)
    for dt_ref in g["dt"]:
        dt = integ.stable_dt(states)
        assert dt == pytest.approx(float(dt_ref), rel=1e-10)
        assert bool(integ.checked_step_inplace(states, dt).view(torch.int32)[0].item())
    err = np.abs(states["hexahedron"][elem, node].cpu().numpy() - g["final"]) / g["final_scale"]
    assert err.max() <= 1e-9, err.max()
    np.testing.assert_allclose(t0, g["totals0"], rtol=0, atol=1e-12 * np.abs(g["totals0"]).max())
    np.testing.assert_allclose(_totals(op, states), g["totals"], rtol=0, atol=1e-12 * np.abs(g["totals0"]).max())
