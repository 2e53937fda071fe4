"""The nodal admissibility certificate of the positivity and troubled-cell kernels
(``nodal_certificate`` in csrc/aux_kernels.cuh; hexahedron and dense kernels), restated in numpy
and checked for soundness: whenever it holds for an element's nodal values, every limiter sample
(nodes, volume points, face points) and the cell mean are admissible, so the kernels may skip the
sample contraction (the troubled kernel) or keep the state as it is (the positivity limiter,
whose theta is then 1).  Also: the Lebesgue constant that the plan derives from the 1-D tables
(``dgb_plan_set_hex``) bounds the row sums sum_i |B_i| of the actual sample basis."""

import numpy as np
import pytest

from jax_fluid_sim_b200 import meshgen
from jax_fluid_sim_b200.mesh import HybridMesh
from jax_fluid_sim_b200.plan import Plan, hex_sumfact_tables

GAMMA = 1.4


def lebesgue_from_tables(plan):
    """The constant dgb_plan_set_hex computes: max(1, L_q^3, L_f^2) over the packed 1-D rows."""
    tables = hex_sumfact_tables(plan)[0]
    P = plan.degree
    N, Q, QF = P + 1, {1: 2, 2: 3, 3: 5}[P], {1: 2, 2: 3, 3: 4}[P]
    bq = tables[:Q * N].reshape(Q, N)
    bf = tables[80:80 + QF * N].reshape(QF, N)
    return max(1.0, np.abs(bq).sum(axis=1).max() ** 3, np.abs(bf).sum(axis=1).max() ** 2)


def certificate(U, L, rho_floor, p_floor, rel):
    if not np.all(np.isfinite(U)):
        return False
    mn, mx = U[:, :5].min(axis=0), U[:, :5].max(axis=0)
    c, h = 0.5 * (mn + mx), 0.5 * (mx - mn)
    a, b = c - L * h, c + L * h
    tol_r = 1e-12 * L * max(abs(a[0]), abs(b[0]))
    if not (a[0] - tol_r > 0.0) or not (a[0] >= 1e-3 * b[0]):
        return False
    m2hi = sum(max(a[d] ** 2, b[d] ** 2) for d in (1, 2, 3))
    m2lo = sum(0.0 if a[d] <= 0.0 <= b[d] else min(a[d] ** 2, b[d] ** 2) for d in (1, 2, 3))
    g1 = GAMMA - 1.0
    ke_hi, ke_lo = 0.5 * m2hi / a[0], 0.5 * m2lo / b[0]
    p_lo, pmean_hi = g1 * (a[4] - ke_hi), g1 * (b[4] - ke_lo)
    tol_p = 1e-6 * g1 * (L * max(abs(a[4]), abs(b[4])) + ke_hi)
    return (a[0] - tol_r >= max(rho_floor, rel * (b[0] + tol_r))) and \
        (p_lo - tol_p >= max(p_floor, rel * pmean_hi + tol_p))


def pressure(S):
    return (GAMMA - 1.0) * (S[..., 4] - 0.5 * (S[..., 1:4] ** 2).sum(axis=-1) / np.maximum(S[..., 0], 1e-14))


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_certificate_is_sound(degree):
    plan = Plan(HybridMesh(meshgen.box_hex((3, 3, 3))), degree)
    bp = plan.blocks[0]
    L = lebesgue_from_tables(plan)
    rows = np.concatenate([np.eye(bp.Np), bp.ref.B, bp.face_sample_B])
    assert L >= np.abs(rows).sum(axis=1).max() * (1 - 1e-14)
    rng = np.random.default_rng(degree)
    base = np.array([1.0, 3.5, 0.3, -0.2, 1.0 / (GAMMA - 1.0) + 0.5 * (3.5 ** 2 + 0.3 ** 2 + 0.2 ** 2)])
    passed = failed = 0
    for trial in range(600):
        amp = 10.0 ** rng.uniform(-4, 0.3)
        U = base[None, :] * (1.0 + amp * rng.standard_normal((bp.Np, 5)))
        S = rows @ U
        w = bp.ref.weights * rng.uniform(0.5, 2.0, bp.Nq)
        mean = w @ (bp.ref.B @ U) / w.sum()
        for rel, rf, pf in ((0.05, 1e-10, 1e-10), (0.0, 1e-10, 1e-10)):
            if certificate(U, L, rf, pf, rel):
                passed += 1
                assert S[:, 0].min() >= max(rf, rel * mean[0])
                assert pressure(S).min() >= max(pf, rel * pressure(mean))
                assert mean[0] >= rf and pressure(mean) >= pf
            else:
                failed += 1
    assert passed > 100 and failed > 100


def test_certificate_refuses_non_finite_values():
    U = np.ones((8, 5))
    U[:, 4] = 3.0
    assert certificate(U, 1.0, 1e-10, 1e-10, 0.05)
    U[3, 2] = np.nan
    assert not certificate(U, 1.0, 1e-10, 1e-10, 0.05)


@pytest.mark.parametrize("etype", ["wedge", "tetra", "hexahedron"])
def test_certificate_is_sound_on_the_dense_sample_rows(etype):
    """The dense kernels take L as the largest row sum of [I; B; B_face] (dgb_plan_set_block): the
    certificate is sound with that L for every element type's sample rows."""
    src = meshgen.hybrid_box((3, 3, 3), seed=5)
    plan = Plan(HybridMesh(src), 2)
    bp = next(b for b in plan.blocks if b.etype == etype) if etype != "hexahedron" else \
        Plan(HybridMesh(meshgen.box_hex((3, 3, 3))), 2).blocks[0]
    rows = np.concatenate([np.eye(bp.Np), bp.ref.B, bp.face_sample_B])
    L = max(1.0, np.abs(np.concatenate([bp.ref.B, bp.face_sample_B])).sum(axis=1).max())
    rng = np.random.default_rng(7)
    base = np.array([1.0, 0.5, -0.3, 0.2, 2.5 + 0.5 * (0.25 + 0.09 + 0.04)])
    passed = 0
    for trial in range(400):
        amp = 10.0 ** rng.uniform(-4, 0.3)
        U = base[None, :] * (1.0 + amp * rng.standard_normal((bp.Np, 5)))
        S = rows @ U
        w = bp.ref.weights * rng.uniform(0.5, 2.0, bp.Nq)
        mean = w @ (bp.ref.B @ U) / w.sum()
        if certificate(U, L, 1e-10, 1e-10, 0.05):
            passed += 1
            assert S[:, 0].min() >= 0.05 * mean[0]
            assert pressure(S).min() >= 0.05 * pressure(mean)
    assert passed > 50
