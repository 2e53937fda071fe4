"""Host-side geometry metrics of plan set-up (``dgb_map_metrics``, csrc/setup.cpp, host threads,
no GPU) against plain numpy: Jacobians, determinants, inverses and w|det J| of curved and
straight elements at shared reference points, with and without an element gather index, and the
face normals and area weights from the mapped tangents (hybrid/geometry.py:139-203, 299-353); and
the subcell face metrics of the MOOD plan (``dgb_subcell_face_metrics``, hybrid/subcell.py:336-360)."""

import numpy as np
import pytest

from jax_fluid_sim_b200 import _native as N
from jax_fluid_sim_b200 import meshgen
from jax_fluid_sim_b200.mesh import HybridMesh
from jax_fluid_sim_b200.reference import RefElement


@pytest.mark.parametrize("degree", [1, 2])
def test_element_metrics_match_numpy(degree):
    geo = RefElement("hexahedron", degree)
    rng = np.random.default_rng(degree)
    E = 700
    xyz = geo.nodes[None] * rng.uniform(0.5, 2.0, (E, 1, 3)) + 0.05 * rng.standard_normal((E, len(geo.nodes), 3))
    pts = RefElement("hexahedron", 3).points
    w = RefElement("hexahedron", 3).weights
    g = geo.basis_gradients(pts)
    index = rng.permutation(E)[:500]
    J, det, inv, wdet = N.map_metrics(xyz, g, index=index, weights=w,
                                      outputs=("jacobian", "det", "inv_jacobian", "wdet"))
    Jr = np.einsum("ekd,qkr->eqdr", xyz[index], g)
    np.testing.assert_allclose(J, Jr, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(det, np.linalg.det(Jr), rtol=1e-12)
    np.testing.assert_allclose(inv, np.linalg.inv(Jr), rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(wdet, w[None] * np.abs(np.linalg.det(Jr)), rtol=1e-12)


def test_face_normals_and_weights_match_numpy():
    mesh = HybridMesh(meshgen.curved_box())
    block = mesh.element_blocks[0]
    geo, xyz = mesh.geometry(block)
    shapes = np.array([[0.25, 0.25, 0.25, 0.25], [0.7, 0.1, 0.1, 0.1], [0.1, 0.1, 0.7, 0.1]])
    corners = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.0, 1.0, 0.0], [0.0, 1.0, 0.0]])
    pts = shapes @ corners
    tu = np.tile([1.0, 0.0, 0.0], (3, 1))
    tv = np.tile([0.0, 1.0, 0.0], (3, 1))
    orient = np.tile([0.0, 0.0, -1.0], (len(xyz), 1))
    qw = np.array([0.5, 0.25, 0.25])
    n, a = N.map_metrics(xyz, geo.basis_gradients(pts), weights=qw, tangents=np.stack([tu, tv], axis=1),
                         orientation=orient, outputs=("normals", "area_weights"))
    J = np.einsum("ekd,qkr->eqdr", xyz, geo.basis_gradients(pts))
    c = np.cross(np.einsum("eqdr,qr->eqd", J, tu), np.einsum("eqdr,qr->eqd", J, tv))
    c *= np.where(np.sum(c * orient[:, None], axis=-1) >= 0, 1.0, -1.0)[..., None]
    mag = np.linalg.norm(c, axis=-1)
    np.testing.assert_allclose(n, c / mag[..., None], rtol=1e-13, atol=1e-14)
    np.testing.assert_allclose(a, qw[None] * mag, rtol=1e-13)
    assert np.all(n[..., 2] < 0)


def test_bad_arguments_are_errors():
    g = RefElement("hexahedron", 1).basis_gradients(np.zeros((1, 3)))
    with pytest.raises(ValueError):
        N.map_metrics(np.zeros((2, 8, 3)), g, outputs=("wdet",))          # wdet needs weights
    with pytest.raises(ValueError):
        N.map_metrics(np.zeros((2, 8, 3)), g, weights=np.ones(1), outputs=("normals",))   # needs tangents
    with pytest.raises(ValueError):
        N.map_metrics(np.zeros((2, 8, 3)), g, index=[0, 2], outputs=("det",))          # index past the nodes


def _subcell_face_metrics_numpy(pv, cen, faces, owners, neighbors):
    """hybrid/subcell.py:336-360 restated with numpy, one face at a time."""
    av, fc = [], []
    for face in faces:
        p = pv[:, np.asarray(face)]
        a = 0.5 * np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
        if len(face) == 4:
            a = a + 0.5 * np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0])
        av.append(a)
        fc.append(p.mean(axis=1))
    av, fc = np.stack(av, axis=1), np.stack(fc, axis=1)
    oc = cen[:, owners]
    d = fc - oc if neighbors is None else cen[:, neighbors] - oc
    av = av * np.where(np.sum(av * d, axis=-1) >= 0.0, 1.0, -1.0)[..., None]
    area = np.linalg.norm(av, axis=-1)
    return av / area[..., None], area, fc


@pytest.mark.parametrize("source", ["hybrid", "curved"])
def test_subcell_face_metrics_match_numpy(source):
    """dgb_subcell_face_metrics (host threads) against the numpy restatement, on the internal and
    boundary subfaces of every element type of a hybrid box and of a curved hexahedron box."""
    from jax_fluid_sim_b200.subcell import ReferenceSubcells
    src = meshgen.hybrid_box((3, 3, 3), seed=4) if source == "hybrid" else meshgen.curved_box()
    mesh = HybridMesh(src)
    for block in mesh.element_blocks:
        rs = ReferenceSubcells(block.element_type)
        geo, xyz = mesh.geometry(block)
        pv = np.einsum("vi,eid->evd", geo.basis(rs.vertices), xyz)
        cen = pv[:, rs.cells].mean(axis=2)
        for faces, own, nbr in ((rs.internal_faces, rs.internal_owner, rs.internal_neighbor),
                                (rs.boundary_faces, rs.boundary_owner, None)):
            got = N.subcell_face_metrics(pv, cen, faces, own, nbr)
            want = _subcell_face_metrics_numpy(pv, cen, faces, own, nbr)
            for g, w in zip(got, want):
                np.testing.assert_allclose(g, w, rtol=1e-13, atol=1e-15)


def test_subcell_face_metrics_reject_bad_faces():
    pv, cen = np.zeros((1, 4, 3)), np.zeros((1, 1, 3))
    with pytest.raises(ValueError):
        N.subcell_face_metrics(pv, cen, [(0, 1)], np.zeros(1, np.int32))          # two vertices
    with pytest.raises(ValueError):
        N.subcell_face_metrics(pv, cen, [(0, 1, 7)], np.zeros(1, np.int32))       # vertex out of range
