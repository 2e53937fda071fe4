"""Host-side geometry metrics of plan set-up (``dgb_map_metrics``, csrc/setup.cpp, host threads,
no GPU) against plain numpy: Jacobians, determinants, inverses and w|det J| of curved and
straight elements at shared reference points, with and without an element gather index, and the
face normals and area weights from the mapped tangents (hybrid/geometry.py:139-203, 299-353)."""

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
