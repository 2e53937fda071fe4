"""The product's face tables against the reference's own outputs (golden fixtures), on the CPU.

``jax_fluid_sim_b200.HybridMesh`` builds the face blocks the kernels read (pairing, owners,
local faces, orientation, tags).  The fixtures hold the reference's ``HybridMesh`` face blocks
(hybrid/mesh.py:361-477) for every golden case, written by ``tests/golden/make_golden.py``.
Integer tables must match bit for bit; normals and areas to 1e-14 of their largest magnitude
(the same float64 cross products, summed in a different order).
"""

import numpy as np
import pytest

from jax_fluid_sim_b200 import HybridMesh

from .conftest import GOLDEN_CASES, load_golden


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_product_face_tables_bit_exact(case):
    g = load_golden(case)
    mesh = HybridMesh(g["source"])
    assert [b.element_type for b in mesh.element_blocks] == list(g["block_names"])
    fixture_types = sorted({k.split("_")[1] for k in g if k.startswith("face_") and k.endswith("_nodes")})
    assert sorted(mesh.face_blocks) == fixture_types
    for ftype, fb in mesh.face_blocks.items():
        for key in ("nodes", "owner_block", "owner_local", "owner_face", "neighbor_block", "neighbor_local",
                    "neighbor_face", "boundary_tags"):
            ours, ref = np.asarray(getattr(fb, key)), g[f"face_{ftype}_{key}"]
            assert ours.shape == ref.shape, (key, ours.shape, ref.shape)
            np.testing.assert_array_equal(ours, ref, err_msg=f"{ftype} {key}")
        for key in ("normals", "areas"):
            ref = g[f"face_{ftype}_{key}"]
            err = np.max(np.abs(np.asarray(getattr(fb, key)) - ref)) / max(np.max(np.abs(ref)), 1e-300)
            assert err <= 1e-14, (ftype, key, err)
