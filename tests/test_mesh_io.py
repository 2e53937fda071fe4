"""Host-side mesh ingestion in the native library: the face pairing (``dgb_pair_faces``) against a
numpy restatement of the reference's pairing order (hybrid/mesh.py:378-459), and the Gmsh ASCII
section parsers (``dgb_msh2_*``, ``dgb_msh4_*``) on well-formed and malformed records.  No GPU."""

import numpy as np
import pytest

from jax_fluid_sim_b200 import _native, gmsh, meshgen


def numpy_pairing(key, visit):
    """Faces in the reference's order: group equal keys (visits in order within a group), then
    internal faces by their second visit and boundary faces by their first."""
    k = key.shape[1]
    srt = np.lexsort((visit,) + tuple(key[:, j] for j in range(k - 1, -1, -1)))
    ks = key[srt]
    new = np.ones(len(ks), bool)
    new[1:] = np.any(ks[1:] != ks[:-1], axis=1)
    gid = np.cumsum(new) - 1
    first = srt[new]
    second = np.full(len(first), -1)
    second[gid[~new]] = srt[~new]
    inner = np.flatnonzero(second >= 0)
    inner = inner[np.argsort(visit[second[inner]], kind="stable")]
    outer = np.flatnonzero(second < 0)
    outer = outer[np.argsort(visit[first[outer]], kind="stable")]
    sel = np.concatenate([inner, outer])
    return first[sel], second[sel]


@pytest.mark.parametrize("n,k,hi,seed", [(0, 4, 5, 0), (1, 3, 5, 1), (9, 4, 3, 2), (5000, 3, 30, 3),
                                         (400000, 4, 80, 4)])
def test_pair_faces_matches_reference_order(n, k, hi, seed):
    rng = np.random.default_rng(seed)
    base = np.unique(np.sort(rng.integers(0, hi, (n // 2 + 1, k)), axis=1), axis=0)
    rows = np.concatenate([base, base[: len(base) // 2]])[:n]
    perm = rng.permutation(len(rows))
    rows = rows[perm]
    visit = (rng.permutation(len(rows)) * 7 + 3).astype(np.int64)
    own, nbr = _native.pair_faces(rows, visit)
    ref_own, ref_nbr = numpy_pairing(rows, visit)
    np.testing.assert_array_equal(own, ref_own)
    np.testing.assert_array_equal(nbr, ref_nbr)


def test_pair_faces_rejects_a_face_of_three_cells():
    with pytest.raises(ValueError, match="more than two cells"):
        _native.pair_faces(np.array([[1, 2, 3]] * 3), np.arange(3))


def test_msh_parsers_read_records():
    body = b"1 0.5 -1.25e-1 +2\n7 1 2 3\n"
    ids, xyz = _native.msh_nodes(body, 2, 2)
    np.testing.assert_array_equal(ids, [1, 7])
    np.testing.assert_array_equal(xyz, [[0.5, -0.125, 2.0], [1.0, 2.0, 3.0]])
    body = b"1 2 2 5 9 1 2 3\r\n2 5 0 1 2 3 4 5 6 7 8\n"
    t, phys, off, nodes = _native.msh_elements(body, 2, 2, 64)
    np.testing.assert_array_equal(t, [2, 5])
    np.testing.assert_array_equal(phys, [5, 0])
    np.testing.assert_array_equal(off, [0, 3, 11])
    np.testing.assert_array_equal(nodes, [1, 2, 3, 1, 2, 3, 4, 5, 6, 7, 8])
    body = b"2 3 1 3\n2 4 0 2\n3\n1\n0 0 0\n1 1 1\n0 1 0 1\n2\n0.5 0 0\n"
    ids, xyz = _native.msh_nodes(body, 3, 4)
    np.testing.assert_array_equal(ids, [3, 1, 2])
    np.testing.assert_array_equal(xyz, [[0, 0, 0], [1, 1, 1], [0.5, 0, 0]])
    body = b"1 2 1 2\n2 6 2 2\n1 1 2 3\n2 2 3 1\n"
    t, dim, tag, off, nodes = _native.msh_elements(body, 2, 4, 64)
    np.testing.assert_array_equal(t, [2, 2])
    np.testing.assert_array_equal(dim, [2, 2])
    np.testing.assert_array_equal(tag, [6, 6])
    np.testing.assert_array_equal(nodes, [1, 2, 3, 2, 3, 1])


@pytest.mark.parametrize("call", [
    lambda: _native.msh_nodes(b"1 0.5 x 2\n", 1, 2),
    lambda: _native.msh_nodes(b"1 0.5\n", 1, 2),
    lambda: _native.msh_elements(b"1 2 2 5\n", 2, 2, 64),
    lambda: _native.msh_elements(b"1 5 0 1 2 3 4 5 6 7 8\n", 1, 2, 4),
    lambda: _native.msh_nodes(b"1 3 1 3\n2 4 0 2\n3\n1\n0 0 0\n1 1 1\n", 3, 4),
    lambda: _native.msh_elements(b"1 3 1 3\n2 6 2 2\n1 1 2 3\n2 2 3 1\n", 3, 4, 64),
])
def test_msh_parsers_reject_malformed_records(call):
    with pytest.raises(ValueError):
        call()


def test_ascii_reader_round_trips_a_sphere_grid(tmp_path):
    from jax_fluid_sim_b200.mesh import HybridMesh
    src = meshgen.sphere_oh_grid(n=4, n_radial=2, outer=((1, 3), (1, 1), (1, 1)))
    path = tmp_path / "s.msh"
    gmsh.write_msh22(path, src)
    back = gmsh.read_msh(path)
    np.testing.assert_array_equal(back.points, src.points)
    assert back.field_data == src.field_data
    ma, mb = HybridMesh(src), HybridMesh(back)
    for ftype, fa in ma.face_blocks.items():
        fb = mb.face_blocks[ftype]
        for key in ("nodes", "owner_block", "owner_local", "neighbor_block", "neighbor_local", "boundary_tags"):
            np.testing.assert_array_equal(getattr(fa, key), getattr(fb, key))
