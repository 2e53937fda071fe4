"""Golden fixture of the reference's aerodynamic force integration (hybrid/aerodynamics.py:149-305),
made by running the reference's own code under the numpy stand-in for JAX.

    python tests/golden/make_golden_aero.py [/path/to/reference]

Case: the box_p2 golden mesh and states (tests/golden/box_p2.npz: jittered hexahedra at P2,
mu = 0.01, isothermal walls at 1.2) with the "walls" boundary as the body, q_inf = 0.5 and the
moment centre (0.2, 0.3, 0.1).  Writes tests/golden/aero_box_p2.npz with the pressure and
viscous forces and moments of the smooth and shocked states and the derived coefficients.
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

# aerodynamics.py imports matplotlib for its history plots, which this fixture does not use
for _name in ("matplotlib", "matplotlib.pyplot"):
    sys.modules.setdefault(_name, types.ModuleType(_name))
sys.modules["matplotlib"].use = lambda *args, **kwargs: None
sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]

import meshio  # noqa: E402  (the stand-in)
import jax.numpy as jnp  # noqa: E402
from hybrid.solver import HybridCompressibleSolver  # noqa: E402
from hybrid.navier_stokes import HybridNavierStokesOperator  # noqa: E402
from hybrid.boundary import FarfieldWallBoundary  # noqa: E402
from hybrid.aerodynamics import AerodynamicForceCalculator  # noqa: E402

from jax_fluid_sim_b200.meshgen import MeshSource  # noqa: E402

KEYS = ("Fx_pressure", "Fy_pressure", "Fz_pressure", "Fx_viscous", "Fy_viscous", "Fz_viscous", "Mx", "My", "Mz",
        "CD", "CL", "CS", "CMx", "CMy", "CMz", "reference_area", "reference_length")


def main():
    with np.load(HERE / "box_p2.npz") as z:
        g = {k: z[k] for k in z.files}
    src = MeshSource.from_arrays(g)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "mesh.msh")
        meshio.write_gmsh22(path, src.points, src.cells, src.physical, src.field_data)
        solver = HybridCompressibleSolver(path, polynomial_degree=int(g["degree"]), dynamic_viscosity=float(g["mu"]),
                                          gamma=1.4, gas_constant=1.0)
    op = HybridNavierStokesOperator(solver)
    bc = FarfieldWallBoundary(solver, jnp.asarray(g["farfield"]), wall_temperature=float(g["wall_temperature"]))
    calc = AerodynamicForceCalculator(op, bc, wall_tag_names=("walls",), moment_center=(0.2, 0.3, 0.1))
    names = [str(n) for n in g["block_names"]]
    out = {}
    for label in ("smooth", "shocked"):
        states = {k: jnp.asarray(g[f"U_{label}_{k}"]) for k in names}
        res = calc.compute(states, q_inf=0.5)
        out[f"{label}"] = np.asarray([getattr(res, k) for k in KEYS], np.float64)
    np.savez_compressed(HERE / "aero_box_p2.npz", keys=np.asarray(KEYS), **out)
    print("wrote aero_box_p2.npz")


if __name__ == "__main__":
    main()
