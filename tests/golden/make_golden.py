"""Generate golden fixtures by running the reference's own hybrid solver.

Run in the build container only (it reads the reference checkout, which does
not exist on the GPU machines):

    python tests/golden/make_golden.py [/path/to/reference]

The reference's ``hybrid/*.py`` files run unmodified under the numpy stand-ins
in ``tests/golden/refshim`` (JAX and meshio are not installable here).  The
``hybrid`` package ``__init__`` is bypassed (it imports matplotlib/GUI code that
is off the path).  Each fixture stores the mesh arrays, the inputs and the
reference outputs; ``tests/test_oracle_golden.py`` pins the oracle to them and
the GPU tests compare the CUDA path to the same numbers.
"""

import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
REFERENCE = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

sys.path.insert(0, str(HERE / "refshim"))
sys.path.insert(0, str(REPO))
_pkg = types.ModuleType("hybrid")
_pkg.__path__ = [str(REFERENCE / "hybrid")]
sys.modules["hybrid"] = _pkg

import meshio  # noqa: E402  (the stand-in)
import jax.numpy as jnp  # noqa: E402
from hybrid.solver import HybridCompressibleSolver  # noqa: E402
from hybrid.navier_stokes import HybridNavierStokesOperator  # noqa: E402
from hybrid.boundary import FarfieldWallBoundary  # noqa: E402
from hybrid.time_integration import HybridSSPRK3  # noqa: E402
from hybrid.limiter import (HybridPositivityLimiter, HybridTroubledCellSensor,  # noqa: E402
                            HybridMOODSubcellLimiter)
from hybrid.subcell import HybridSubcellFV  # noqa: E402

from jax_fluid_sim_b200 import meshgen  # noqa: E402


def smooth_primitive(xyz):
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    rho = 1.0 + 0.2 * np.sin(2 * x + y) * np.cos(z)
    u = 0.5 + 0.1 * np.cos(x + 2 * z)
    v = 0.2 * np.sin(y)
    w = -0.1 * np.cos(x)
    p = 1.0 + 0.1 * np.sin(x + y + z)
    return np.stack([rho, u, v, w, p], axis=-1)


def shocked_primitive(xyz, x_shock):
    W = smooth_primitive(xyz)
    behind = xyz[..., 0] < x_shock
    W[..., 0] = np.where(behind, 3.0 * W[..., 0], W[..., 0])
    W[..., 4] = np.where(behind, 6.0 * W[..., 4], W[..., 4])
    W[..., 1] = np.where(behind, W[..., 1] + 1.0, W[..., 1])
    return W


def run_case(name, source, degree, mu, farfield, wall_temperature, x_shock, mood=False, step=True, species=()):
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "mesh.msh")
        meshio.write_gmsh22(path, source.points, source.cells, source.physical, source.field_data)
        solver = HybridCompressibleSolver(path, polynomial_degree=degree, dynamic_viscosity=mu,
                                          gamma=1.4, gas_constant=1.0, species_names=tuple(species))
    op = HybridNavierStokesOperator(solver)
    bc = FarfieldWallBoundary(solver, jnp.asarray(farfield), wall_temperature=wall_temperature)
    geo = op.geometry
    names = [b.element_type for b in solver.mesh.element_blocks]
    out["block_names"] = np.asarray(names)
    for ftype, fb in solver.mesh.face_blocks.items():
        for key in ("nodes", "owner_block", "owner_local", "owner_face", "neighbor_block",
                    "neighbor_local", "neighbor_face", "normals", "areas", "boundary_tags"):
            out[f"face_{ftype}_{key}"] = np.asarray(getattr(fb, key))
        fm = geo.face_metrics[ftype]
        out[f"face_{ftype}_qnormals"] = np.asarray(fm.normals)
        out[f"face_{ftype}_qweights"] = np.asarray(fm.integration_weights)
        out[f"face_{ftype}_owner_points"] = np.asarray(fm.owner_reference_points)
        out[f"face_{ftype}_neighbor_points"] = np.asarray(fm.neighbor_reference_points)
    for b, block in enumerate(solver.mesh.element_blocks):
        m = geo.element_metrics[b]
        out[f"elem_{block.element_type}_wdet"] = np.asarray(m.integration_weights)
        out[f"elem_{block.element_type}_minv"] = np.asarray(m.inverse_mass_matrix)
    xyz = geo.solution_node_coordinates
    smooth = {k: np.asarray(solver.primitive_to_conserved(jnp.asarray(smooth_primitive(np.asarray(xyz[k])))))
              for k in names}
    shocked = {k: np.asarray(solver.primitive_to_conserved(jnp.asarray(shocked_primitive(np.asarray(xyz[k]), x_shock))))
               for k in names}
    for k in names:
        out[f"xyz_{k}"] = np.asarray(xyz[k])
        out[f"U_smooth_{k}"] = smooth[k]
        out[f"U_shocked_{k}"] = shocked[k]
    for label, states in (("smooth", smooth), ("shocked", shocked)):
        s = {k: jnp.asarray(v) for k, v in states.items()}
        inv = op.inviscid_rhs(s, bc)
        vis = op.viscous_rhs(s, bc)
        for k in names:
            out[f"rhs_inviscid_{label}_{k}"] = np.asarray(inv[k])
            out[f"rhs_viscous_{label}_{k}"] = np.asarray(vis[k])
        positivity = HybridPositivityLimiter(op)
        sensor = HybridTroubledCellSensor(op)
        integ = HybridSSPRK3(op, cfl=0.3, limiter=positivity)
        out[f"dt_{label}"] = np.asarray(integ.stable_dt(s, bc))
        values, flags = sensor(s)
        lim = positivity(s)
        for k in names:
            out[f"sensor_{label}_{k}"] = np.asarray(values[k])
            out[f"limited_{label}_{k}"] = np.asarray(lim[k])
        mood_lim = HybridMOODSubcellLimiter(op, positivity=positivity)
        tr = mood_lim.troubled(s)
        for k in names:
            out[f"troubled_{label}_{k}"] = np.asarray(tr[k])
        if step:
            dt = float(out[f"dt_{label}"])
            res, valid, rmin, pmin = integ.checked_step(s, dt, bc)
            out[f"step_{label}_valid"] = np.asarray(valid)
            out[f"step_{label}_rho_min"] = np.asarray(rmin)
            out[f"step_{label}_p_min"] = np.asarray(pmin)
            for k in names:
                out[f"step_{label}_{k}"] = np.asarray(res[k])
    if mood:
        # MOOD subcell recompute with the detected flags, each reconstruction, and a full
        # checked SSP-RK3 step with the MOOD limiter (time_integration.py:450-554)
        s = {k: jnp.asarray(v) for k, v in shocked.items()}
        dt = float(out["dt_shocked"])
        inv = op.inviscid_rhs(s, bc)
        vis = op.viscous_rhs(s, bc)
        cand = {k: s[k] + dt * (inv[k] + vis[k]) for k in names}
        positivity = HybridPositivityLimiter(op)
        mood_lim = HybridMOODSubcellLimiter(op, positivity=positivity)
        tr = mood_lim.troubled(cand)
        for k in names:
            out[f"mood_troubled_{k}"] = np.asarray(tr[k])
        for recon in ("constant", "tvd", "weno"):
            sub = HybridSubcellFV(op, reconstruction=recon)
            res = sub.recompute(s, cand, dt, tr, boundary_state=bc, additional_rhs=vis)
            for k in names:
                out[f"mood_{recon}_{k}"] = np.asarray(res[k])
        integ = HybridSSPRK3(op, cfl=0.3, limiter=mood_lim)
        res, valid, rmin, pmin = integ.checked_step(s, dt, bc)
        out["mood_step_valid"] = np.asarray(valid)
        out["mood_step_rho_min"] = np.asarray(rmin)
        for k in names:
            out[f"mood_step_{k}"] = np.asarray(res[k])
    if species:
        out["species"] = np.asarray(species)
    out["degree"] = np.asarray(degree)
    out["mu"] = np.asarray(mu)
    out["farfield"] = np.asarray(farfield, float)
    out["wall_temperature"] = np.asarray(np.nan if wall_temperature is None else wall_temperature)
    source.save(HERE / f"{name}.npz", **out)
    print(f"wrote {name}.npz")


def main():
    ff = [1.0, 0.6, 0.1, 0.0, 1.0]
    for p in (1, 2, 3):
        run_case(f"smoke_p{p}", meshgen.smoke_mesh(), p, 0.02, ff, None, 0.5)
    box = meshgen.box_hex((3, 3, 2), lo=(0, 0, 0), hi=(1.5, 1.5, 1.0), jitter=0.15, seed=7)
    for p in (2, 3):
        run_case(f"box_p{p}", box, p, 0.01, ff, 1.2, 0.6, mood=True)
    run_case("mixed_p2", meshgen.mixed_block(jitter=0.1, seed=3), 2, 0.01, ff, 1.1, 1.0, mood=True)
    run_case("curved_p2", meshgen.curved_box(amplitude=0.05), 2, 0.01, ff, 1.2, 0.6, mood=True)


if __name__ == "__main__":
    main()
