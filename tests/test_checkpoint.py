"""Restart files in the reference driver's format (run_hybrid_sphere.py:36-45,123-131): keys,
dtypes and values round-trip; in-place loading keeps the buffers; on the GPU a run resumed from
a restart file continues bit-identically to the uninterrupted run."""

import numpy as np
import pytest
import torch

from jax_fluid_sim_b200.checkpoint import load_restart, save_restart


def test_round_trip_matches_reference_layout(tmp_path):
    rng = np.random.default_rng(0)
    states = {"hexahedron": torch.as_tensor(rng.random((5, 27, 5))), "tetra": torch.as_tensor(rng.random((3, 10, 5)))}
    path = tmp_path / "checkpoint_latest.npz"
    save_restart(path, states, 0.125, 42)
    with np.load(path) as z:
        assert sorted(z.files) == ["U_hexahedron", "U_tetra", "step", "time"]
        assert z["U_hexahedron"].dtype == np.float64 and z["time"].shape == () and int(z["step"]) == 42
    assert not (tmp_path / "checkpoint_latest.tmp.npz").exists()
    loaded, t, step = load_restart(path, device="cpu")
    assert t == 0.125 and step == 42
    for k in states:
        np.testing.assert_array_equal(loaded[k].numpy(), states[k].numpy())
    buf = {k: torch.zeros_like(v) for k, v in states.items()}
    ptrs = {k: v.data_ptr() for k, v in buf.items()}
    again, _, _ = load_restart(path, into=buf)
    for k in states:
        assert again[k].data_ptr() == ptrs[k]
        np.testing.assert_array_equal(again[k].numpy(), states[k].numpy())
    with pytest.raises(KeyError):
        load_restart(path, element_types=["wedge"], device="cpu")
    with pytest.raises(ValueError):
        load_restart(path, into={"tetra": torch.zeros((4, 10, 5), dtype=torch.float64)})


def test_missing_step_defaults_to_zero(tmp_path):
    path = tmp_path / "old.npz"
    np.savez_compressed(path, time=np.asarray(1.5), U_hexahedron=np.ones((2, 8, 5)))
    states, t, step = load_restart(path, device="cpu")
    assert t == 1.5 and step == 0 and states["hexahedron"].shape == (2, 8, 5)


@pytest.mark.gpu
def test_resumed_graph_run_continues_bit_identically(tmp_path):
    """Three graph-replayed MOOD steps on the smallest sphere grid, against one step, a restart
    file written from the device buffers, the buffers overwritten and reloaded in place, and two
    more steps (the captured graph is reused: same pointers, same dt)."""
    import jax_fluid_sim_b200 as jfs
    from jax_fluid_sim_b200 import workloads
    solver, op, bc, coupler, start = workloads.reacting_case("tiny", degree=2)
    lim = jfs.HybridMOODSubcellLimiter(op, positivity=jfs.HybridPositivityLimiter(op))
    integ = jfs.HybridSSPRK3(op, cfl=0.3, limiter=lim, graph=True)
    dt = integ.stable_dt(start, bc)
    ref = {k: v.clone() for k, v in start.items()}
    for _ in range(3):
        integ.checked_step_inplace(ref, dt, bc)
    U = {k: v.clone() for k, v in start.items()}
    integ.checked_step_inplace(U, dt, bc)
    save_restart(tmp_path / "r.npz", U, dt, 1)
    for v in U.values():
        v.fill_(float("nan"))
    U2, t, step = load_restart(tmp_path / "r.npz", into=U)
    assert step == 1 and t == dt and all(U2[k].data_ptr() == U[k].data_ptr() for k in U)
    for _ in range(2):
        integ.checked_step_inplace(U, dt, bc)
    for k in ref:
        assert torch.equal(U[k], ref[k])
