"""CUDA path vs the reference's own outputs (golden fixtures) through the C ABI.

Tolerances: float64 everywhere; the kernels sum in a different order than the
reference's einsums, so values agree to a relative 1e-9 of each field's largest
magnitude.  Face connectivity and troubled-cell flags must match exactly.
"""

import numpy as np
import pytest
import torch

from .conftest import GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu
RTOL = 1e-9


def close(a, b, rtol=RTOL):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a, float)
    b = np.asarray(b, float)
    scale = max(np.max(np.abs(b)), 1e-300)
    err = np.max(np.abs(a - b)) / scale
    assert err <= rtol, f"relative error {err:.3e} > {rtol:.1e}"
    return True


def setup(case):
    """case may carry a ':dense' suffix to force the generic dense path on a hexahedron mesh."""
    from jax_fluid_sim_b200 import (FarfieldWallBoundary, HybridCompressibleSolver, HybridMesh,
                                    HybridNavierStokesOperator)
    name, _, path = case.partition(":")
    g = load_golden(name)
    solver = HybridCompressibleSolver(HybridMesh(g["source"]), polynomial_degree=int(g["degree"]),
                                      dynamic_viscosity=float(g["mu"]),
                                      species_names=tuple(str(n) for n in g.get("species", ())))
    op = HybridNavierStokesOperator(solver, sum_factorised=False if path == "dense" else None)
    wt = float(g["wall_temperature"])
    bc = FarfieldWallBoundary(solver, g["farfield"], wall_temperature=None if np.isnan(wt) else wt)
    return g, solver, op, bc


CASES = GOLDEN_CASES + ["box_p2:dense", "box_p3:dense", "species_p2:dense", "curved_p2:dense"]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("label", ["smooth", "shocked"])
def test_rhs_matches_reference(case, label):
    g, solver, op, bc = setup(case)
    states = {k: g[f"U_{label}_{k}"] for k in g["block_names"]}
    inv = op.inviscid_rhs(states, bc)
    vis = op.viscous_rhs(states, bc)
    for k in g["block_names"]:
        close(inv[k], g[f"rhs_inviscid_{label}_{k}"])
        close(vis[k], g[f"rhs_viscous_{label}_{k}"])


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("label", ["smooth", "shocked"])
def test_dt_limiter_flags_step(case, label):
    from jax_fluid_sim_b200 import (HybridMOODSubcellLimiter, HybridPositivityLimiter, HybridSSPRK3,
                                    HybridTroubledCellSensor)
    g, solver, op, bc = setup(case)
    states = {k: g[f"U_{label}_{k}"] for k in g["block_names"]}
    pos = HybridPositivityLimiter(op)
    integ = HybridSSPRK3(op, cfl=0.3, limiter=pos)
    close(integ.stable_dt(states, bc), g[f"dt_{label}"], 1e-12)
    values, _ = HybridTroubledCellSensor(op)(states)
    lim = pos(states)
    troubled = HybridMOODSubcellLimiter(op, positivity=pos).troubled(states)
    for k in g["block_names"]:
        close(values[k], g[f"sensor_{label}_{k}"], 1e-9)
        close(lim[k], g[f"limited_{label}_{k}"])
        np.testing.assert_array_equal(troubled[k].cpu().numpy(), g[f"troubled_{label}_{k}"])
    res, valid, rmin, pmin = integ.checked_step(states, float(g[f"dt_{label}"]), bc)
    assert valid == bool(g[f"step_{label}_valid"])
    close(rmin, g[f"step_{label}_rho_min"], 1e-9)
    close(pmin, g[f"step_{label}_p_min"], 1e-9)
    for k in g["block_names"]:
        close(res[k], g[f"step_{label}_{k}"], 1e-9)


@pytest.mark.parametrize("case", ["smoke_p2", "box_p2", "box_p3:dense"])
@pytest.mark.parametrize("poison", [0, 4, 1])
def test_dt_of_nan_state_matches_reference(case, poison):
    """A NaN in one node's density, energy or momentum makes the reference's rate NaN, which
    stable_dt maps to 1e7 (jnp.maximum keeps NaN through the 1e-14 floors,
    hybrid/time_integration.py:107-108,167).  With cfl = 5 the result 5e-7 lies inside the clip
    range, so a kernel that dropped the NaN at a floor (a huge finite rate, clipped to 1e-7)
    fails."""
    from jax_fluid_sim_b200 import HybridSSPRK3
    from oracle.dg import TimeIntegrator

    from .test_oracle_golden import build as oracle_build
    g, solver, op, bc = setup(case)
    states = {k: np.array(g[f"U_smooth_{k}"]) for k in g["block_names"]}
    first = g["block_names"][0]
    states[first][0, 0, poison] = np.nan
    expected = TimeIntegrator(oracle_build(case.partition(":")[0])[2], cfl=5.0).stable_dt(states)
    assert abs(expected - 5e-7) <= 1e-18, expected
    close(HybridSSPRK3(op, cfl=5.0).stable_dt(states, bc), expected, 1e-12)


def test_uniform_state_is_steady():
    """A uniform state with no boundary ghost has an exactly zero inviscid residual (anchor form)."""
    from jax_fluid_sim_b200 import HybridCompressibleSolver, HybridMesh, HybridNavierStokesOperator
    from jax_fluid_sim_b200 import meshgen
    solver = HybridCompressibleSolver(HybridMesh(meshgen.box_hex((3, 3, 3), periodic=(True, True, True))),
                                      polynomial_degree=3, dynamic_viscosity=0.01)
    op = HybridNavierStokesOperator(solver)
    U = solver.uniform_state_blocks(1.0, [2.0, 0.3, -0.1], 3.5)
    r = op.inviscid_rhs(U)
    assert torch.count_nonzero(r["hexahedron"]).item() == 0


@pytest.mark.parametrize("case", ["box_p3", "smoke_p3", "mixed_p2", "box_p3:dense", "curved_p2:dense"])
def test_device_inverse_mass_matches_host(case):
    """The inverse mass matrices built on the device (dgb_plan_build_inverse_mass: M = B^T
    diag(w|J|) B in shared memory, Gauss-Jordan elimination) give the residual of the numpy-inverted
    host copies to round-off (1e-12 relative), on the sum-factorised (transposed) and the dense
    path.  The affine shortcut is off, so every element reads its own matrix."""
    from jax_fluid_sim_b200.operators import NativePlan
    g, solver, op, bc = setup(case)
    states = {k: g[f"U_shocked_{k}"] for k in g["block_names"]}
    out = []
    for where in ("device", "host"):
        other = object.__new__(type(op))
        other.__dict__.update({k: v for k, v in op.__dict__.items() if k != "native"})
        other.native = NativePlan(op.plan, solver, op.viscous, op.br2_stabilization, op.native.sum_factorised,
                                  "float64", affine=False, inverse_mass=where)
        out.append(other.rhs(states, bc))
    for k in g["block_names"]:
        close(out[0][k], out[1][k].cpu().numpy(), 1e-12)


def test_degenerate_element_is_refused_by_the_device_inverse_mass():
    """A block whose w|J| are all zero has a singular mass matrix: the device build reports it."""
    from jax_fluid_sim_b200.operators import NativePlan
    g, solver, op, bc = setup("box_p2")
    bp = op.plan.blocks[0]
    saved = bp.wdet
    bp.wdet = np.zeros_like(saved)
    try:
        with pytest.raises(ValueError, match="positive definite"):
            NativePlan(op.plan, solver, op.viscous, op.br2_stabilization, True, "float64")
    finally:
        bp.wdet = saved


MOOD_CASES = ["box_p2", "box_p3", "mixed_p2", "box_p2:dense", "species_p2", "species_p2:dense", "curved_p2",
              "curved_p2:dense"]


@pytest.mark.parametrize("case", MOOD_CASES)
def test_mood_recompute_and_step(case):
    """MOOD subcell recompute (constant / TVD / CWENO-Z) and the MOOD checked step vs the reference."""
    from jax_fluid_sim_b200 import (HybridMOODSubcellLimiter, HybridPositivityLimiter, HybridSSPRK3,
                                    HybridSubcellFV)
    g, solver, op, bc = setup(case)
    s = {k: g[f"U_shocked_{k}"] for k in g["block_names"]}
    dt = float(g["dt_shocked"])
    inv = op.inviscid_rhs(s, bc)
    vis = op.viscous_rhs(s, bc)
    U = op.to_device(s)
    cand = {k: U[k] + dt * (inv[k] + vis[k]) for k in U}
    pos = HybridPositivityLimiter(op)
    lim = HybridMOODSubcellLimiter(op, positivity=pos)
    tr = lim.troubled(cand)
    for k in g["block_names"]:
        np.testing.assert_array_equal(tr[k].cpu().numpy(), g[f"mood_troubled_{k}"])
    for recon in ("constant", "tvd", "weno"):
        res = HybridSubcellFV(op, reconstruction=recon).recompute(s, cand, dt, tr, bc, vis)
        for k in g["block_names"]:
            close(res[k], g[f"mood_{recon}_{k}"])
    integ = HybridSSPRK3(op, cfl=0.3, limiter=lim)
    res, valid, rmin, pmin = integ.checked_step(s, dt, bc)
    assert valid == bool(g["mood_step_valid"])
    for k in g["block_names"]:
        close(res[k], g[f"mood_step_{k}"])


@pytest.mark.parametrize("case", ["box_p2", "box_p3", "mixed_p2", "smoke_p1", "smoke_p3", "box_p2:dense", "species_p2",
                                  "curved_p2"])
@pytest.mark.parametrize("label", ["smooth", "shocked"])
def test_mixed_precision_against_reference(case, label):
    """precision='mixed' (float32 trace, lift, volume and finalize arithmetic, on the
    sum-factorised hexahedron path and on the dense path of hexahedra, prisms and tetrahedra)
    against the reference's float64 residuals: within 2e-5 of each field's largest magnitude, and
    one checked step within the 1e-6 relative density L2 gate of the float64 step."""
    from jax_fluid_sim_b200 import HybridPositivityLimiter, HybridSSPRK3
    g, solver, op, bc = setup(case)
    mixed = op.with_precision("mixed")
    states = {k: g[f"U_{label}_{k}"] for k in g["block_names"]}
    inv, vis = mixed.inviscid_rhs(states, bc), mixed.viscous_rhs(states, bc)
    for k in g["block_names"]:
        close(inv[k], g[f"rhs_inviscid_{label}_{k}"], 2e-5)
        close(vis[k], g[f"rhs_viscous_{label}_{k}"], 2e-5)
    dt = HybridSSPRK3(op, cfl=0.3).stable_dt(states, bc)
    plain = HybridSSPRK3(op, cfl=0.3, limiter=HybridPositivityLimiter(op)).checked_step(states, dt, bc)[0]
    step = HybridSSPRK3(mixed, cfl=0.3, limiter=HybridPositivityLimiter(mixed)).checked_step(states, dt, bc)[0]
    num = sum(float(((step[k][..., 0] - plain[k][..., 0]) ** 2).sum()) for k in plain)
    den = sum(float((plain[k][..., 0] ** 2).sum()) for k in plain)
    assert (num / den) ** 0.5 <= 1e-6
