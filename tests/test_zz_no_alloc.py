"""The allocation-free time-step entry point against the planned one.

dgb_stable_dt_noalloc serves callers that may not allocate device memory while they
run (a host code or coupling framework that owns a fixed device-memory pool, or a time
loop that must not call cudaMalloc); its scratch is a static device array.  This test
calls it through the C ABI twice in a row, on two different states and sizes, and checks
each result against dgb_stable_dt of a full plan.  It is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(n, degree, mu, seed):
    import jax_fluid_sim_b200 as jfs
    from jax_fluid_sim_b200 import meshgen
    src = meshgen.box_hex(n, hi=(1.5, 1.0, 1.2), jitter=0.1, seed=seed)
    solver = jfs.HybridCompressibleSolver(jfs.HybridMesh(src), polynomial_degree=degree, dynamic_viscosity=mu)
    op = jfs.HybridNavierStokesOperator(solver)
    xyz = op.solution_node_coordinates["hexahedron"]
    rng = np.random.default_rng(seed)
    W = np.stack([1.0 + 0.3 * np.sin(4 * xyz[..., 0]) + 0.05 * rng.random(xyz.shape[:-1]),
                  0.8 * np.cos(3 * xyz[..., 1]), 0.2 + 0 * xyz[..., 0], -0.4 * np.sin(xyz[..., 2]),
                  1.0 + 0.4 * np.cos(2 * xyz[..., 0] * xyz[..., 1])], -1)
    return solver, op, {"hexahedron": solver.primitive_to_conserved(W)}


def test_noalloc_dt_matches_planned_dt_twice():
    from jax_fluid_sim_b200 import HybridSSPRK3
    from jax_fluid_sim_b200 import _native as N
    L = N.lib()
    # a viscous P3 case, then an inviscid P2 one on another mesh; both cfl values put the
    # expected dt well inside the clip range (1e-7, 1e-3), so the rates are really compared
    for n, degree, mu, seed, cfl in (((4, 3, 3), 3, 0.01, 1, 0.3), ((6, 5, 2), 2, 0.0, 2, 0.05)):
        solver, op, U = _case(n, degree, mu, seed)
        integ = HybridSSPRK3(op, cfl=cfl)
        expected = integ.stable_dt(U)
        assert 2e-7 < expected < 0.9e-3, expected
        Ud = op.to_device(U)["hexahedron"]
        length = torch.as_tensor(op.plan.blocks[0].length, device="cuda")
        dt = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        E, Np, nv = Ud.shape
        rc = L.dgb_stable_dt_noalloc(Ud.data_ptr(), length.data_ptr(), E, Np, nv, degree, solver.gamma,
                                     solver.gas_constant, solver.dynamic_viscosity, solver.thermal_conductivity,
                                     op.br2_stabilization, cfl, dt.data_ptr(),
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, L.dgb_noalloc_last_error()
        got = float(dt.item())
        assert abs(got - expected) <= 1e-12 * abs(expected), (got, expected)


def test_noalloc_nan_state_gives_reference_rate():
    """A NaN density in one node: the reference maps that element's NaN rate to 1e7, so with
    cfl = 5 the step is 5e-7, the same as the planned entry point's."""
    from jax_fluid_sim_b200 import HybridSSPRK3
    from jax_fluid_sim_b200 import _native as N
    L = N.lib()
    solver, op, U = _case((4, 3, 3), 2, 0.01, 3)
    U["hexahedron"][2, 5, 0] = np.nan
    expected = HybridSSPRK3(op, cfl=5.0).stable_dt(U)
    assert abs(expected - 5e-7) <= 1e-18, expected
    Ud = op.to_device(U)["hexahedron"]
    length = torch.as_tensor(op.plan.blocks[0].length, device="cuda")
    dt = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    E, Np, nv = Ud.shape
    rc = L.dgb_stable_dt_noalloc(Ud.data_ptr(), length.data_ptr(), E, Np, nv, 2, solver.gamma, solver.gas_constant,
                                 solver.dynamic_viscosity, solver.thermal_conductivity, op.br2_stabilization, 5.0,
                                 dt.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.dgb_noalloc_last_error()
    assert abs(float(dt.item()) - expected) <= 1e-12 * expected


def test_noalloc_rejects_oversized_blocks():
    from jax_fluid_sim_b200 import _native as N
    L = N.lib()
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = L.dgb_stable_dt_noalloc(dummy.data_ptr(), dummy.data_ptr(), (1 << 20) + 1, 8, 5, 1, 1.4, 1.0, 0.0, 0.0,
                                 3.0, 0.3, dummy.data_ptr(), None)
    assert rc == -1
    assert b"at most 1048576 elements" in L.dgb_noalloc_last_error()
    rc = L.dgb_stable_dt_noalloc(dummy.data_ptr(), dummy.data_ptr(), 1, 8, 5, -1, 1.4, 1.0, 0.0, 0.0,
                                 3.0, 0.3, dummy.data_ptr(), None)
    assert rc == -1
    assert b"degree" in L.dgb_noalloc_last_error()
