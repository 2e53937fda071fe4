"""The tensor-core (tcgen05, three-term TF32) inviscid volume kernel of the prism and tetrahedron
blocks against the oracle and against the CUDA-core kernels, through the C ABI.

Case: the conforming hexahedron/prism/tetrahedron box of the vortex study, (4, 3, 4) cubes
jittered 10 %, at P1-P3, Euler.  The hexahedra keep the CUDA-core dense kernel (64 nodes at P3
exceed the tensor-core kernel's shared memory), so every residual below mixes both kernels.

Tolerance: 4e-4 of each field's largest magnitude against the oracle's float64 residual and
against the CUDA-core mixed kernel (observed: 5e-6 at P1, 1e-4 at P2, 2.6e-4 at P3 in the
tetrahedron block).  Each operand is held as two rounded TF32 terms, about 2^-22 relative
(float32: 2^-24), and the volume residual is a sum of terms several hundred times larger than
itself (the CUDA-core float32 kernel shows 2e-5 here at P3), so the bound is several times the
float32 one.  One checked step stays within the mixed-precision gate (density 1e-6
relative L2 against the float64 step) and conserves mass, momentum and energy to 1e-9 relative.
No device error may be recorded (every wait in the kernel is bounded)."""

import numpy as np
import pytest
import torch

from jax_fluid_sim_b200 import HybridSSPRK3, workloads

pytestmark = pytest.mark.gpu


def _close(a, b, tol):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    scale = max(np.max(np.abs(b)), 1e-300)
    err = np.max(np.abs(a - b)) / scale
    assert err <= tol, f"relative error {err:.3e} > {tol:.1e}"
    return err


def _case(degree, affine=True):
    from jax_fluid_sim_b200 import HybridCompressibleSolver, HybridEulerOperator, meshgen
    from jax_fluid_sim_b200.mesh import HybridMesh
    from oracle.dg import Operator
    from oracle.mesh import Mesh, MeshSource
    from oracle.physics import Gas
    src = meshgen.hybrid_box((4, 3, 4), jitter=0.1, seed=1)
    solver = HybridCompressibleSolver(HybridMesh(src), polynomial_degree=degree)
    op = HybridEulerOperator(solver, precision="mixed", affine=affine)
    states = solver.state_blocks_from_primitive_function(op, lambda x: workloads.vortex_primitive(x, radius=0.2))
    mesh = Mesh(MeshSource(src.points, src.cells, src.physical, src.field_data, src.periodic_map))
    return solver, op, states, Operator(mesh, Gas(), degree)


@pytest.mark.parametrize("degree", [1, 2, 3])
@pytest.mark.parametrize("affine", [True, False])
def test_tensor_core_residual_against_oracle(degree, affine):
    solver, op, states, oop = _case(degree, affine)
    cuda_cores = op.rhs(states)
    # the prism and the tetrahedron block (and at P1 the hexahedra: 8 nodes, 8 points)
    assert op.native.set_tensor_cores(True) == (3 if degree == 1 else 2)
    got = op.rhs(states)
    assert op.native.device_errors() == 0
    U = {k: v.detach().cpu().numpy() for k, v in states.items()}
    ref = oop.inviscid_rhs(U)
    for k in U:
        _close(got[k], ref[k], 4e-4)
        _close(got[k], cuda_cores[k].cpu().numpy(), 4e-4)
    assert op.native.set_tensor_cores(False) == 0
    again = op.rhs(states)
    for k in U:
        assert torch.equal(again[k], cuda_cores[k])


def test_tensor_core_step_against_oracle():
    """One checked SSP-RK3 step at P3 through the captured graph: density within 1e-6 (relative
    L2) of the oracle's float64 step, and mass, momentum and energy conserved to 1e-9."""
    from oracle.dg import TimeIntegrator
    solver, op, states, oop = _case(3)
    assert op.native.set_tensor_cores(True) == 2
    U = {k: v.detach().cpu().numpy() for k, v in states.items()}
    oint = TimeIntegrator(oop, cfl=0.3)
    dt = oint.stable_dt(U)
    ref = oint.checked_step(U, dt)[0]
    cur = {k: v.clone() for k, v in states.items()}
    status = HybridSSPRK3(op, cfl=0.3, graph=True).checked_step_inplace(cur, dt)
    assert bool(status.view(torch.int32)[0].item())
    assert op.native.device_errors() == 0
    num = sum(np.sum((cur[k][..., 0].cpu().numpy() - ref[k][..., 0]) ** 2) for k in U)
    den = sum(np.sum(ref[k][..., 0] ** 2) for k in U)
    assert np.sqrt(num / den) <= 1e-6
    t0, t1 = _totals(op, U), _totals(op, {k: v.cpu().numpy() for k, v in cur.items()})
    assert np.all(np.abs(t1 - t0) <= 1e-9 * np.abs(t0).max())


def _totals(op, states):
    out = np.zeros(5)
    for name, bp in zip(op.names, op.plan.blocks):
        out += np.einsum("eq,qn,env->v", bp.wdet, bp.ref.B, states[name])
    return out
