"""Pin the CPU oracle to the reference's own outputs (golden fixtures).

The fixtures were produced by ``tests/golden/make_golden.py`` running the
reference's ``hybrid/`` code.  Connectivity, tags and troubled flags must match
exactly; floating-point outputs to the stated relative tolerance (float64 with
different summation order).
"""

import numpy as np
import pytest

from oracle.dg import Operator, PositivityLimiter, TimeIntegrator, TroubledCellSensor, mood_troubled
from oracle.mesh import Mesh, MeshSource
from oracle.physics import FarfieldWallBoundary, Gas

from .conftest import GOLDEN_CASES, load_golden

RTOL = 1e-9          # float64 restatement vs reference, relative to the field's max magnitude


def close(a, b, rtol=RTOL):
    a, b = np.asarray(a, float), np.asarray(b, float)
    scale = max(np.max(np.abs(b)), 1e-300)
    return np.max(np.abs(a - b)) <= rtol * scale


def build(case):
    g = load_golden(case)
    src = MeshSource(g["source"].points, g["source"].cells, g["source"].physical, g["source"].field_data,
                     g["source"].periodic_map)
    mesh = Mesh(src)
    gas = Gas(dynamic_viscosity=float(g["mu"]), n_species=len(g["species"]) if "species" in g else 0)
    op = Operator(mesh, gas, int(g["degree"]))
    wt = float(g["wall_temperature"])
    bc = FarfieldWallBoundary(gas, mesh.physical_names, g["farfield"], wall_temperature=None if np.isnan(wt) else wt)
    return g, mesh, op, bc


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_connectivity_bit_exact(case):
    g, mesh, op, _ = build(case)
    assert list(g["block_names"]) == [b.element_type for b in mesh.element_blocks]
    for ftype, fb in mesh.face_blocks.items():
        for key in ("nodes", "owner_block", "owner_local", "owner_face", "neighbor_block",
                    "neighbor_local", "neighbor_face", "boundary_tags"):
            np.testing.assert_array_equal(getattr(fb, key), g[f"face_{ftype}_{key}"], err_msg=key)
        assert close(fb.normals, g[f"face_{ftype}_normals"], 1e-14)
        fm = op.geo.face[ftype]
        np.testing.assert_array_equal(fm.owner_points, g[f"face_{ftype}_owner_points"])
        np.testing.assert_array_equal(np.nan_to_num(fm.neighbor_points, nan=-7.0),
                                      np.nan_to_num(g[f"face_{ftype}_neighbor_points"], nan=-7.0))
        assert close(fm.normals, g[f"face_{ftype}_qnormals"], 1e-13)
        assert close(fm.weights, g[f"face_{ftype}_qweights"], 1e-13)


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_element_metrics(case):
    g, mesh, op, _ = build(case)
    for k, b in enumerate(mesh.element_blocks):
        assert close(op.geo.element[k].wdet, g[f"elem_{b.element_type}_wdet"], 1e-13)
        assert close(op.geo.element[k].minv, g[f"elem_{b.element_type}_minv"], 1e-10)


@pytest.mark.parametrize("case", GOLDEN_CASES)
@pytest.mark.parametrize("label", ["smooth", "shocked"])
def test_rhs(case, label):
    g, mesh, op, bc = build(case)
    states = {k: g[f"U_{label}_{k}"] for k in g["block_names"]}
    inv = op.inviscid_rhs(states, bc)
    vis = op.viscous_rhs(states, bc)
    for k in g["block_names"]:
        assert close(inv[k], g[f"rhs_inviscid_{label}_{k}"]), k
        assert close(vis[k], g[f"rhs_viscous_{label}_{k}"]), k


@pytest.mark.parametrize("case", GOLDEN_CASES)
@pytest.mark.parametrize("label", ["smooth", "shocked"])
def test_dt_limiter_sensor_step(case, label):
    g, mesh, op, bc = build(case)
    states = {k: g[f"U_{label}_{k}"] for k in g["block_names"]}
    pos = PositivityLimiter(op)
    integ = TimeIntegrator(op, cfl=0.3, limiter=pos)
    dt = integ.stable_dt(states)
    assert close(dt, g[f"dt_{label}"], 1e-12)
    values, flags = TroubledCellSensor(op)(states)
    lim = pos(states)
    troubled = mood_troubled(op, pos, TroubledCellSensor(op), states)
    for k in g["block_names"]:
        assert close(values[k], g[f"sensor_{label}_{k}"], 1e-9)
        assert close(lim[k], g[f"limited_{label}_{k}"])
        np.testing.assert_array_equal(troubled[k], g[f"troubled_{label}_{k}"])
    res, valid, rmin, pmin = integ.checked_step(states, float(g[f"dt_{label}"]), bc)
    assert valid == bool(g[f"step_{label}_valid"])
    assert close(rmin, g[f"step_{label}_rho_min"], 1e-9)
    for k in g["block_names"]:
        assert close(res[k], g[f"step_{label}_{k}"], 1e-9)


MOOD_CASES = ["box_p2", "box_p3", "mixed_p2", "species_p2", "curved_p2"]


@pytest.mark.parametrize("case", MOOD_CASES)
def test_mood_recompute_and_step(case):
    from oracle.subcell import MOODLimiter, SubcellFV
    g, mesh, op, bc = build(case)
    s = {k: g[f"U_shocked_{k}"] for k in g["block_names"]}
    dt = float(g["dt_shocked"])
    inv = op.inviscid_rhs(s, bc)
    vis = op.viscous_rhs(s, bc)
    cand = {k: s[k] + dt * (inv[k] + vis[k]) for k in s}
    pos = PositivityLimiter(op)
    lim = MOODLimiter(op, positivity=pos)
    tr = lim.troubled(cand)
    for k in g["block_names"]:
        np.testing.assert_array_equal(tr[k], g[f"mood_troubled_{k}"])
    for recon in ("constant", "tvd", "weno"):
        res = SubcellFV(op, reconstruction=recon).recompute(s, cand, dt, tr, bc, vis)
        for k in g["block_names"]:
            assert close(res[k], g[f"mood_{recon}_{k}"]), (recon, k)
    integ = TimeIntegrator(op, cfl=0.3, limiter=lim)
    res, valid, rmin, pmin = integ.checked_step(s, dt, bc)
    assert valid == bool(g["mood_step_valid"])
    for k in g["block_names"]:
        assert close(res[k], g[f"mood_step_{k}"]), k
