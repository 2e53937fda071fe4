"""Wall forces and moments (dgb_wall_forces) against the reference's own AerodynamicForceCalculator
run on the box_p2 golden case (tests/golden/aero_box_p2.npz, make_golden_aero.py): the "walls"
boundary as the body, q_inf 0.5, moment centre (0.2, 0.3, 0.1), smooth and shocked states.

Tolerance: 1e-9 of the largest force or moment component (float64, different summation order;
the reference anchors its pressure traces on the cell mean, these on the first node)."""

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = np.load(Path(__file__).resolve().parent / "golden" / "aero_box_p2.npz")


@pytest.mark.parametrize("label", ["smooth", "shocked"])
def test_wall_forces_match_reference(label):
    from jax_fluid_sim_b200.aerodynamics import AerodynamicForceCalculator
    from .test_gpu_parity import setup
    g, solver, op, bc = setup("box_p2")
    calc = AerodynamicForceCalculator(op, bc, wall_tag_names=("walls",), moment_center=(0.2, 0.3, 0.1))
    states = {k: g[f"U_{label}_{k}"] for k in g["block_names"]}
    res = calc.compute(states, q_inf=0.5)
    ref = dict(zip([str(k) for k in GOLDEN["keys"]], GOLDEN[label]))
    scale = max(abs(ref[k]) for k in ("Fx_pressure", "Fy_pressure", "Fz_pressure", "Fx_viscous", "Fy_viscous",
                                      "Fz_viscous", "Mx", "My", "Mz"))
    qa = 0.5 * ref["reference_area"]
    for k, v in ref.items():
        if k in ("reference_area", "reference_length"):
            tol = 1e-12 * abs(v)
        elif k.startswith("CM"):
            tol = 1e-9 * scale / (qa * ref["reference_length"])
        elif k.startswith("C"):
            tol = 1e-9 * scale / qa
        else:
            tol = 1e-9 * scale
        assert abs(getattr(res, k) - v) <= tol, (k, getattr(res, k), v)


def test_linear_pressure_gives_the_enclosed_volume_force():
    """A closed body in p = p0 + G . x with the fluid at rest: the pressure force on it is
    -G V (Gauss), V the volume the wall faces enclose, and there is no viscous force.  On the
    smallest sphere grid at P2 the traces are exact for linear p."""
    import jax_fluid_sim_b200 as jfs
    from jax_fluid_sim_b200 import meshgen
    from jax_fluid_sim_b200.aerodynamics import AerodynamicForceCalculator, face_points
    src = meshgen.sphere_oh_grid(n=4, n_radial=2, outer=((1, 3), (1, 1), (1, 1)))
    solver = jfs.HybridCompressibleSolver(jfs.HybridMesh(src), polynomial_degree=2, dynamic_viscosity=1e-3)
    op = jfs.HybridNavierStokesOperator(solver)
    G = np.array([0.3, -0.2, 0.1])
    bc = jfs.FarfieldWallBoundary(solver, np.array([1.0, 0.0, 0.0, 0.0, 1.0]), wall_temperature=1.0)

    def prim(x):
        W = np.zeros(x.shape[:-1] + (5,))
        W[..., 0] = 1.0 + 0.0 * x[..., 0]
        W[..., 4] = 2.0 + x @ G
        return W

    states = solver.state_blocks_from_primitive_function(op, prim)
    calc = AerodynamicForceCalculator(op, bc)
    out = calc.forces_device(states).cpu().numpy()
    # enclosed volume by the divergence theorem over the wall faces (normals point into the body)
    fp = op.plan.faces["quad"]
    wall = (fp.nbr_block < 0) & np.isin(fp.tags, calc.wall_tags)
    x = face_points(op.plan)["quad"][wall]
    V = -np.sum(np.einsum("fqd,fqd->fq", x, fp.normals[wall]) * fp.weights[wall]) / 3.0
    assert 0.4 < V < 0.53                       # the faceted sphere of radius 0.5
    np.testing.assert_allclose(out[0:3], -G * V, rtol=0, atol=1e-11)
    np.testing.assert_allclose(out[6:9], 0.0, atol=1e-11)
