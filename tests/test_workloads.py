"""Host-side checks of the benchmark workloads: the periodic conforming hybrid box and the
closed-form initial states (Taylor-Green and isentropic vortex)."""

import numpy as np
import pytest

from jax_fluid_sim_b200 import meshgen, workloads
from jax_fluid_sim_b200.mesh import HybridMesh
from jax_fluid_sim_b200.plan import Plan, _p1_jacobian
from oracle.mesh import Mesh, MeshSource


@pytest.mark.parametrize("n,seed", [((4, 3, 4), 1), ((6, 5, 7), 4), ((8, 8, 8), 0)])
def test_hybrid_box_is_conforming_and_periodic(n, seed):
    src = meshgen.hybrid_box(n, jitter=0.1, seed=seed)
    mesh = HybridMesh(src)
    assert all(int(np.sum(fb.neighbor_block < 0)) == 0 for fb in mesh.face_blocks.values())
    plan = Plan(mesh, 1)
    assert sum(bp.volume.sum() for bp in plan.blocks) == pytest.approx(1.0, rel=1e-13)
    for bp, block in zip(plan.blocks, mesh.element_blocks):
        J = _p1_jacobian(bp.etype, mesh.points[block.connectivity][:, None], bp.ref.points[None])
        assert np.all(np.linalg.det(J) > 0.0), bp.etype
    frac = meshgen.hybrid_box_fractions(src)
    assert set(frac) == {"hexahedron", "wedge", "tetra"} and all(0.1 < f < 0.6 for f in frac.values())


def test_hybrid_box_faces_match_oracle_pairing():
    """Face pairing, owners and orientations of the periodic box bit-exact against the oracle."""
    src = meshgen.hybrid_box((4, 3, 4), jitter=0.1, seed=2)
    ours = HybridMesh(src)
    ref = Mesh(MeshSource(src.points, src.cells, src.physical, src.field_data, src.periodic_map))
    assert [b.element_type for b in ours.element_blocks] == [b.element_type for b in ref.element_blocks]
    for ftype, fb in ours.face_blocks.items():
        rb = ref.face_blocks[ftype]
        for key in ("nodes", "owner_block", "owner_local", "owner_face", "neighbor_block", "neighbor_local",
                    "neighbor_face"):
            np.testing.assert_array_equal(getattr(fb, key), getattr(rb, key), err_msg=key)
        np.testing.assert_allclose(fb.normals, rb.normals, rtol=0, atol=1e-14)


def test_hybrid_box_is_seeded_and_checks_size():
    a, b = meshgen.hybrid_box((4, 4, 4), seed=3), meshgen.hybrid_box((4, 4, 4), seed=3)
    np.testing.assert_array_equal(a.points, b.points)
    for (na, ca), (nb, cb) in zip(a.cells, b.cells):
        assert na == nb
        np.testing.assert_array_equal(ca, cb)
    with pytest.raises(ValueError):
        meshgen.hybrid_box((2, 4, 4))


def test_vortex_returns_after_one_period():
    rng = np.random.default_rng(0)
    x = rng.random((500, 3))
    T = workloads.vortex_period()
    np.testing.assert_allclose(workloads.vortex_primitive(x, T), workloads.vortex_primitive(x, 0.0), atol=1e-12)
    W = workloads.vortex_primitive(x, 0.3 * T)
    assert np.all(W[:, 0] > 0.0) and np.all(W[:, 4] > 0.0)
    far = workloads.vortex_primitive(np.array([[0.0, 0.0, 0.5]]))[0]
    np.testing.assert_allclose(far[1:4], workloads.vortex_velocity(), atol=1e-6)
    # isentropic: p / rho^gamma is the free-stream value everywhere
    np.testing.assert_allclose(W[:, 4] / W[:, 0] ** 1.4, 1.0, rtol=1e-12)


def test_tgv_initial_state():
    x = np.random.default_rng(1).random((200, 3)) * 2 * np.pi
    W = workloads.tgv_primitive(x)
    assert np.all(W[:, 0] == 1.0) and np.all(W[:, 3] == 0.0)
    assert W[:, 4].min() >= 1.0 / (1.4 * 0.01) - 0.375 - 1e-12
    # divergence-free velocity: du/dx + dv/dy = cos x cos y cos z - cos x cos y cos z
    h = 1e-6
    e = np.eye(3) * h
    div = ((workloads.tgv_primitive(x + e[0])[:, 1] - workloads.tgv_primitive(x - e[0])[:, 1])
           + (workloads.tgv_primitive(x + e[1])[:, 2] - workloads.tgv_primitive(x - e[1])[:, 2])) / (2 * h)
    assert np.max(np.abs(div)) < 1e-8


def test_block_affine_data_equals_dense_tables():
    """Affine elements of the dense path: coef * inv(B^T diag(w) B) equals the per-element
    sliver-scaled inverse mass matrix, w * det equals w |J| and the constant J^-1 equals every
    point's, on the jittered hybrid box (tetrahedra and z-prisms are affine there)."""
    from jax_fluid_sim_b200.plan import block_affine_data
    plan = Plan(HybridMesh(meshgen.hybrid_box((4, 3, 4), jitter=0.1, seed=1)), 2)
    seen = 0
    for bp in plan.blocks:
        aff, coef, jinv, det, w, mref_inv = block_affine_data(bp)
        idx = np.flatnonzero(aff)
        if bp.etype == "tetra":
            assert len(idx) == bp.E
        seen += len(idx)
        for e in idx:
            np.testing.assert_allclose(coef[e] * mref_inv, bp.minv[e], rtol=1e-11, atol=1e-11 * np.abs(bp.minv[e]).max())
            np.testing.assert_allclose(w * det[e], bp.wdet[e], rtol=1e-12)
            np.testing.assert_allclose(np.broadcast_to(jinv[e], (bp.Nq, 9)), bp.jinv[e].reshape(bp.Nq, 9),
                                       rtol=0, atol=1e-12 * np.abs(jinv[e]).max())
    assert seen > 0


def test_cylinder_grid_and_union():
    """The extruded O-grid is valid (positive Jacobians, tagged boundary faces only on the wall,
    the outer ring and the span planes); the union keeps every case's cells in case order."""
    a, b = meshgen.cylinder_o_grid(16, 6), meshgen.cylinder_o_grid(20, 5, outer_radius=8.0)
    mesh = HybridMesh(a)
    quads = mesh.face_blocks["quad"]
    tags = quads.boundary_tags[quads.neighbor_block < 0]
    names = {v: k for k, v in mesh.physical_names.items()}
    assert sorted({names[t] for t in tags}) == ["cylinder_wall", "inlet", "outlet", "symmetry"]
    assert int(np.sum(tags == mesh.physical_names["cylinder_wall"])) == 16
    assert int(np.sum(tags == mesh.physical_names["symmetry"])) == 2 * 16 * 6
    plan = Plan(mesh, 1)
    J = _p1_jacobian("hexahedron", mesh.points[mesh.element_blocks[0].connectivity][:, None],
                     plan.blocks[0].ref.points[None])
    assert np.all(np.linalg.det(J) > 0.0)
    u, counts = meshgen.union([a, b])
    assert counts == [{"hexahedron": 96, "quad": 16 + 16 + 2 * 96}, {"hexahedron": 100, "quad": 20 + 20 + 2 * 100}]
    merged = HybridMesh(u)
    conn = merged.element_blocks[0].connectivity
    np.testing.assert_array_equal(conn[:96], a.cells[0][1])
    np.testing.assert_array_equal(conn[96:], b.cells[0][1] + len(a.points))


def test_ensemble_cases_are_seeded_and_in_range():
    c1, c2 = workloads.ensemble_cases(16, seed=3), workloads.ensemble_cases(16, seed=3)
    assert c1 == c2
    for c in c1:
        assert 0.3 <= c["mach"] <= 4.0 and 1e2 <= c["reynolds"] <= 1e5 and c["degree"] in (2, 3)
        assert 0.6 * 5000 <= c["n_theta"] * c["n_radial"] <= 1.3 * 60000
