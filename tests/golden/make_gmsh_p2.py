"""Extract small Gmsh fixtures of complete second-order hexahedra (Gmsh element type 12) from two
meshes the reference ships, both written by Gmsh itself: mesh/cylinder_conformal_ogrid.msh
(MSH 2.2) and mesh/sphere_aerospace_oh_grid.msh (MSH 4.1).  The first cells of type 12 of each
file are written, with their nodes renumbered 1..n and each cell's node list in the order Gmsh
wrote it, as a small MSH 2.2 file.  These pin the Gmsh node numbering of hexahedron27 against
files from Gmsh rather than against this package's own writer.

    python tests/golden/make_gmsh_p2.py [/path/to/reference]
"""

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from jax_fluid_sim_b200 import gmsh  # noqa: E402

CELLS = 24


def extract(src, dst, label):
    lines = Path(src).read_text().splitlines()
    sec = gmsh._sections(lines)
    version = sec["MeshFormat"][0].split()[0]
    reader = gmsh._read_v2 if version.startswith("2") else gmsh._read_v4
    points, index, records = reader(sec, None)
    cells = np.concatenate([nodes for etype, _, nodes in records if etype == 12])[:CELLS]
    used, inverse = np.unique(cells, return_inverse=True)
    inverse = inverse.reshape(cells.shape)
    xyz = points[index[used]]
    out = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", "1", f'3 1 "{label}"', "$EndPhysicalNames",
           "$Nodes", str(len(xyz))]
    out += [f"{i + 1} {x!r} {y!r} {z!r}" for i, (x, y, z) in enumerate(xyz.tolist())]
    out += ["$EndNodes", "$Elements", str(len(cells))]
    out += [f"{k + 1} 12 2 1 1 " + " ".join(str(int(v) + 1) for v in row) for k, row in enumerate(inverse)]
    out.append("$EndElements")
    Path(dst).write_text("\n".join(out) + "\n")
    print(dst, len(cells), "cells from", src, "(MSH", version + ")")


if __name__ == "__main__":
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    extract(ref / "mesh" / "cylinder_conformal_ogrid.msh", HERE / "gmsh_hex27_cylinder.msh", "fluid")
    extract(ref / "mesh" / "sphere_aerospace_oh_grid.msh", HERE / "gmsh_hex27_sphere.msh", "fluid")
