"""Gmsh MSH 2.2 (ASCII and binary) / 4.1 ASCII reading: a written file reads back to the same mesh
(points, cells, physical tags and names, hence the same face tables), hand-written 4.1 and
second-order files parse, complete second-order cells come back in meshio's node order, and a
binary file written by Gmsh itself parses."""

import numpy as np
import pytest

from jax_fluid_sim_b200 import gmsh, meshgen
from jax_fluid_sim_b200.mesh import HybridMesh


def _same_faces(a, b):
    ma, mb = HybridMesh(a), HybridMesh(b)
    assert [x.element_type for x in ma.element_blocks] == [x.element_type for x in mb.element_blocks]
    for ftype, fa in ma.face_blocks.items():
        fb = mb.face_blocks[ftype]
        for key in ("nodes", "owner_block", "owner_local", "neighbor_block", "neighbor_local", "boundary_tags"):
            np.testing.assert_array_equal(getattr(fa, key), getattr(fb, key))


@pytest.mark.parametrize("source", [meshgen.mixed_block(jitter=0.1, seed=3), meshgen.smoke_mesh()])
def test_msh22_round_trip(tmp_path, source):
    path = tmp_path / "m.msh"
    gmsh.write_msh22(path, source)
    back = gmsh.read_msh(path)
    np.testing.assert_array_equal(back.points, source.points)
    assert back.field_data == source.field_data
    _same_faces(source, back)


@pytest.mark.parametrize("source", [meshgen.mixed_block(jitter=0.1, seed=3), meshgen.smoke_mesh()])
def test_msh22_binary_round_trip(tmp_path, source):
    path = tmp_path / "m.msh"
    gmsh.write_msh22(path, source, binary=True)
    assert path.read_bytes().startswith(b"$MeshFormat\n2.2 1 8\n")
    back = gmsh.read_msh(path)
    np.testing.assert_array_equal(back.points, source.points)
    assert back.field_data == source.field_data
    # the reader groups cells by (type, physical tag), so compare each type's cells as a set
    got = dict(back.cells)
    for ctype, conn in source.cells:
        np.testing.assert_array_equal(np.unique(got[ctype], axis=0), np.unique(conn, axis=0))
    _same_faces(source, back)


def test_msh22_binary_written_by_gmsh(tmp_path):
    """A slice of the reference's binary mesh mesh/sr71_pure_hex.msh (tests/golden/make_gmsh_binary.py:
    600 hexahedra, the 120 boundary quadrilaterals among their nodes, 1,902 nodes, records as Gmsh
    wrote them): counts, names and tags, positive cell volumes, and the same mesh as its ASCII
    rewrite."""
    from pathlib import Path
    from jax_fluid_sim_b200.mesh import _cell_geometry
    src = gmsh.read_msh(Path(__file__).parent / "golden" / "gmsh_sr71_binary.msh")
    assert len(src.points) == 1902
    kinds = dict(src.cells)
    assert len(kinds["hexahedron"]) == 600 and len(kinds["quad"]) == 120
    assert {"inlet", "outlet", "walls", "airfoil_wall", "fluid"} <= set(src.field_data)
    assert np.all(src.physical[0] == src.field_data["fluid"][0])
    surface = {v[0] for v in src.field_data.values() if v[1] == 2}
    assert set(np.unique(src.physical[1]).tolist()) <= surface
    _, vol = _cell_geometry(np.asarray(src.points), "hexahedron", kinds["hexahedron"])
    assert np.all(vol > 0.0)
    path = tmp_path / "ascii.msh"
    gmsh.write_msh22(path, src)
    back = gmsh.read_msh(path)
    np.testing.assert_array_equal(back.points, src.points)
    for (ta, ca), (tb, cb), pa, pb in zip(src.cells, back.cells, src.physical, back.physical):
        assert ta == tb
        np.testing.assert_array_equal(ca, cb)
        np.testing.assert_array_equal(pa, pb)


def test_reference_shim_writer_reads_back(tmp_path):
    """The MSH 2.2 writer the golden fixtures use (tests/golden/refshim/meshio.py) reads back."""
    import importlib.util
    from pathlib import Path
    spec = importlib.util.spec_from_file_location("shim_meshio", Path(__file__).parent / "golden" / "refshim" / "meshio.py")
    shim = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(shim)
    src = meshgen.box_hex((3, 3, 2), lo=(0, 0, 0), hi=(1.5, 1.5, 1.0), jitter=0.15, seed=7)
    path = tmp_path / "b.msh"
    shim.write_gmsh22(str(path), src.points, src.cells, src.physical, src.field_data)
    _same_faces(src, gmsh.read_msh(path))


MSH41 = """$MeshFormat
4.1 0 8
$EndMeshFormat
$PhysicalNames
2
2 7 "walls"
3 1 "fluid"
$EndPhysicalNames
$Entities
0 0 1 1
3 0 0 0 1 1 1 1 7 0
5 0 0 0 1 1 1 1 1 0
$EndEntities
$Nodes
1 8 1 8
3 5 0 8
1
2
3
4
5
6
7
8
0 0 0
1 0 0
1 1 0
0 1 0
0 0 1
1 0 1
1 1 1
0 1 1
$EndNodes
$Elements
2 2 1 2
2 3 3 1
1 1 2 3 4
3 5 5 1
2 1 2 3 4 5 6 7 8
$EndElements
"""


def test_msh41_entities_and_blocks(tmp_path):
    path = tmp_path / "c.msh"
    path.write_text(MSH41)
    src = gmsh.read_msh(path)
    assert src.field_data == {"walls": (7, 2), "fluid": (1, 3)}
    assert [c[0] for c in src.cells] == ["hexahedron", "quad"]
    np.testing.assert_array_equal(src.cells[0][1], [[0, 1, 2, 3, 4, 5, 6, 7]])
    assert src.physical[0].tolist() == [1] and src.physical[1].tolist() == [7]


def test_second_order_cells(tmp_path):
    """Serendipity hexahedron20 keeps its corners."""
    pts = "\n".join(f"{i + 1} {x} {y} {z}" for i, (x, y, z) in enumerate(
        [(a, b, c) for c in (0, 1, 2) for b in (0, 1, 2) for a in (0, 1, 2)]))
    corners = [1, 3, 9, 7, 19, 21, 27, 25]
    hex20 = corners + list(range(2, 14))
    body = f"$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n27\n{pts}\n$EndNodes\n$Elements\n1\n1 17 2 1 1 " + \
           " ".join(map(str, hex20)) + "\n$EndElements\n"
    path = tmp_path / "h20.msh"
    path.write_text(body)
    src = gmsh.read_msh(path)
    np.testing.assert_array_equal(src.cells[0][1][0], np.asarray(corners) - 1)


def _p2_node_deviation(points, meshio_cells):
    """Largest distance, relative to the cell's bounding-box diagonal, between a hexahedron27's
    nodes (taken to the reference element's order by the P2 permutation) and the trilinear map of
    its corners at the reference nodes: small for any cell of a mildly curved mesh, about half the
    cell when the node order is wrong."""
    from jax_fluid_sim_b200.mesh import P2_PERMUTATIONS
    from jax_fluid_sim_b200.reference import RefElement
    ref1, ref2 = RefElement("hexahedron", 1), RefElement("hexahedron", 2)
    xyz = points[meshio_cells[:, P2_PERMUTATIONS["hexahedron27"]]]
    corners = points[meshio_cells[:, :8]]
    linear = np.einsum("ri,eid->erd", ref1.basis(ref2.nodes), corners)
    size = np.linalg.norm(corners.max(axis=1) - corners.min(axis=1), axis=-1)
    return float((np.linalg.norm(xyz - linear, axis=-1).max(axis=1) / size).max())


@pytest.mark.parametrize("name", ["cylinder", "sphere"])
def test_gmsh_hexahedron27_node_order(name):
    """Hexahedron27 cells written by Gmsh (extracted from the reference's own meshes by
    tests/golden/make_gmsh_p2.py) read into meshio's order: every node then sits where the
    reference element puts it (within the cell's curvature), the Jacobian is positive, and the
    unconverted Gmsh order fails the same check."""
    from pathlib import Path
    from jax_fluid_sim_b200.mesh import P2_PERMUTATIONS
    from jax_fluid_sim_b200.reference import RefElement
    path = Path(__file__).parent / "golden" / f"gmsh_hex27_{name}.msh"
    src = gmsh.read_msh(path)
    (ctype, cells), = src.cells
    assert ctype == "hexahedron27" and cells.shape == (24, 27)
    assert _p2_node_deviation(src.points, cells) < 0.01
    ref2 = RefElement("hexahedron", 2)
    J = np.einsum("eid,qir->eqdr", src.points[cells[:, P2_PERMUTATIONS["hexahedron27"]]],
                  ref2.basis_gradients(ref2.points))
    assert np.linalg.det(J).min() > 0.0
    raw = np.empty_like(cells)
    raw[:, gmsh.gmsh_to_meshio("hexahedron27")] = cells       # undo the reordering
    assert _p2_node_deviation(src.points, raw) > 0.3


def test_gmsh_second_order_orders_are_permutations():
    """The Gmsh -> meshio column orders are permutations that keep the corners in place; the
    wedge18 order is the identity (the reference's P2 table takes wedge18 in Gmsh's numbering)."""
    for ctype, n in (("tetra10", 10), ("wedge18", 18), ("hexahedron27", 27)):
        order = gmsh.gmsh_to_meshio(ctype)
        np.testing.assert_array_equal(np.sort(order), np.arange(n))
        corners = {"tetra10": 4, "wedge18": 6, "hexahedron27": 8}[ctype]
        np.testing.assert_array_equal(order[:corners], np.arange(corners))
    np.testing.assert_array_equal(gmsh.gmsh_to_meshio("wedge18"), np.arange(18))


def test_curved_round_trip_and_geometry(tmp_path):
    """A curved hexahedron27 box written as MSH 2.2 (Gmsh order) reads back to the same cells in
    meshio order, and the mesh built from the file has the same element geometry."""
    src = meshgen.curved_box()
    path = tmp_path / "curved.msh"
    gmsh.write_msh22(path, src)
    back = gmsh.read_msh(path)
    volume = lambda m: [np.asarray(c) for t, c in m.cells if t == "hexahedron27"]
    np.testing.assert_array_equal(volume(back)[0], volume(src)[0])
    ma, mb = HybridMesh(src), HybridMesh(back)
    np.testing.assert_array_equal(ma.geometry(ma.element_blocks[0])[1], mb.geometry(mb.element_blocks[0])[1])
    _same_faces(src, back)


def test_hybrid_mesh_and_solver_take_a_path(tmp_path):
    """HybridMesh(path) and HybridCompressibleSolver(path) read the file, as the reference's do."""
    from jax_fluid_sim_b200 import HybridCompressibleSolver
    src = meshgen.mixed_block(jitter=0.1, seed=3)
    path = tmp_path / "mixed.msh"
    gmsh.write_msh22(path, src)
    _same_faces(src, HybridMesh(str(path)).source)
    solver = HybridCompressibleSolver(str(path), polynomial_degree=2)
    assert [b.element_type for b in solver.mesh.element_blocks] == ["hexahedron", "wedge", "tetra"]


def test_msh41_hexahedron27_reads_like_msh22(tmp_path):
    """The same Gmsh-written hexahedron27 cells, written again as MSH 4.1 (one entity, one node
    block, one element block), read to the same meshio-ordered cells as the MSH 2.2 fixture."""
    from pathlib import Path
    src22 = gmsh.read_msh(Path(__file__).parent / "golden" / "gmsh_hex27_cylinder.msh")
    raw = Path(__file__).parent / "golden" / "gmsh_hex27_cylinder.msh"
    lines = raw.read_text().splitlines()
    nodes = lines[lines.index("$Nodes") + 2:lines.index("$EndNodes")]
    elems = lines[lines.index("$Elements") + 2:lines.index("$EndElements")]
    n = len(nodes)
    out = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat", "$PhysicalNames", "1", '3 1 "fluid"', "$EndPhysicalNames",
           "$Entities", "0 0 0 1", "1 -9 -9 -9 9 9 9 1 1 0", "$EndEntities",
           "$Nodes", f"1 {n} 1 {n}", f"3 1 0 {n}"]
    out += [ln.split()[0] for ln in nodes]
    out += [" ".join(ln.split()[1:]) for ln in nodes]
    out += ["$EndNodes", "$Elements", f"1 {len(elems)} 1 {len(elems)}", f"3 1 12 {len(elems)}"]
    out += [" ".join([ln.split()[0]] + ln.split()[5:]) for ln in elems]
    out.append("$EndElements")
    path = tmp_path / "hex27_v41.msh"
    path.write_text("\n".join(out) + "\n")
    src41 = gmsh.read_msh(path)
    np.testing.assert_array_equal(src41.points, src22.points)
    (c41, a41), = src41.cells
    (c22, a22), = src22.cells
    assert c41 == c22 == "hexahedron27"
    np.testing.assert_array_equal(a41, a22)
