"""Learned troubled-cell predictor kernels against the numpy oracle, and its hooks in the step.

Tolerances: features to 1e-5 relative (float32 outputs of float64 statistics); inference to
2e-4 in probability (float16 weights); the training gradient to 1e-4 relative + 1e-7
absolute (float32 atomics in a different summation order).  With the predictor attached in
evaluate mode, or never firing, the MOOD step must be bit-identical to the plain one.
"""

import numpy as np
import pytest
import torch

from oracle import mlp

from .test_gpu_parity import setup

pytestmark = pytest.mark.gpu


def _states(g, label):
    return {k: g[f"U_{label}_{k}"] for k in g["block_names"]}


@pytest.mark.parametrize("case", ["box_p3", "mixed_p2"])
def test_features_match_oracle(case):
    from jax_fluid_sim_b200.predictor import TroubledCellPredictor
    g, solver, op, bc = setup(case)
    states = _states(g, "shocked")
    got = TroubledCellPredictor(op).features(states).cpu().numpy()
    exp = mlp.features(op.plan, states, solver.gamma)
    np.testing.assert_allclose(got, exp, rtol=1e-5, atol=1e-5)


def test_inference_and_gradient_match_oracle():
    from jax_fluid_sim_b200.predictor import TroubledCellPredictor
    g, solver, op, bc = setup("box_p2")
    pred = TroubledCellPredictor(op, seed=3)
    rng = np.random.default_rng(1)
    X = rng.normal(0, 1, (300, 8)).astype(np.float32)
    y = (rng.random(300) < 0.2).astype(np.uint8)
    norm = np.concatenate([rng.normal(0, 0.5, 8), 0.5 + rng.random(8)]).astype(np.float32)
    pred.norm.copy_(torch.as_tensor(norm))
    w16 = pred.weights16.float().cpu().numpy()
    p = pred.predict(torch.as_tensor(X)).cpu().numpy()
    np.testing.assert_allclose(p, mlp.forward(w16, norm, X)[0], atol=2e-4)
    # one Adam step with lr = 0 leaves the weights and exposes the gradient as m / (1 - beta1)
    from jax_fluid_sim_b200 import _native as N
    from jax_fluid_sim_b200.operators import _stream_ptr
    from jax_fluid_sim_b200.predictor import _lib, _ptr
    w0 = pred.weights.cpu().numpy().copy()
    Xd, yd = torch.as_tensor(X).cuda(), torch.as_tensor(y).cuda()
    idx = torch.arange(300, dtype=torch.int32, device="cuda")
    N.check(_lib().dgb_mlp_train_step(_ptr(pred.weights), _ptr(pred.grad), _ptr(pred.m), _ptr(pred.v), None,
                                      _ptr(pred.norm), _ptr(Xd), _ptr(yd), _ptr(idx), 300, 4.0, 0.0, 1, None,
                                      _stream_ptr()))
    gg = pred.m.cpu().numpy() / 0.1
    ge = mlp.gradient(w0, norm, X, y, 4.0)
    assert np.all(pred.grad.cpu().numpy() == 0.0)
    np.testing.assert_array_equal(pred.weights.cpu().numpy(), w0)
    np.testing.assert_allclose(gg, ge, rtol=1e-4, atol=1e-7)


def test_training_separates_a_learnable_rule():
    """Labels = (feature 0 > 0.5): a few epochs must reach > 97 % accuracy."""
    from jax_fluid_sim_b200.predictor import TroubledCellPredictor, confusion
    g, solver, op, bc = setup("box_p2")
    pred = TroubledCellPredictor(op, seed=0)
    rng = np.random.default_rng(2)
    X = rng.normal(0, 1, (20000, 8)).astype(np.float32)
    y = (X[:, 0] > 0.5).astype(np.uint8)
    hist = pred.fit(torch.as_tensor(X), torch.as_tensor(y), epochs=8, batch=1024, lr=3e-3)
    assert hist[-1] < hist[0]
    c = confusion(pred.predict(torch.as_tensor(X)).cpu().numpy() > 0.5, y)
    assert c["missed_rate"] < 0.03 and c["false_positive_rate"] < 0.03


def _mood_step(op, states, bc, dt, predictor=None, mode="off"):
    """One checked MOOD step from ``states``; with a predictor attached in ``mode``, also
    returns its counters for the step."""
    from jax_fluid_sim_b200 import HybridMOODSubcellLimiter, HybridPositivityLimiter, HybridSSPRK3
    lim = HybridMOODSubcellLimiter(op, positivity=HybridPositivityLimiter(op))
    integ = HybridSSPRK3(op, cfl=0.3, limiter=lim)
    U = op.to_device({k: np.array(v, copy=True) for k, v in states.items()})
    if predictor is None:
        integ.checked_step_inplace(U, dt, bc)
        return U, None
    predictor.attach(mode)
    predictor.counts(reset=True)
    integ.checked_step_inplace(U, dt, bc)
    counts = predictor.counts(reset=True)
    predictor.attach("off")
    return U, counts


@pytest.mark.parametrize("case", ["box_p3", "mixed_p2"])
def test_predictor_hooks_in_the_mood_step(case):
    from jax_fluid_sim_b200 import HybridSSPRK3
    from jax_fluid_sim_b200.predictor import TroubledCellPredictor
    g, solver, op, bc = setup(case)
    states = _states(g, "shocked")
    dt = HybridSSPRK3(op, cfl=0.3).stable_dt(states, bc)
    plain, _ = _mood_step(op, states, bc, dt)
    pred = TroubledCellPredictor(op, seed=5)
    # evaluate mode: the plain step, with the prediction only counted
    ev, counts = _mood_step(op, states, bc, dt, pred, "evaluate")
    for k in plain:
        assert torch.equal(ev[k], plain[k])
    assert counts["hit"] + counts["false_positive"] == counts["predicted"]
    # a predictor that never fires leaves the learned step identical to the plain one
    pred.threshold = 2.0
    never, counts = _mood_step(op, states, bc, dt, pred, "learned")
    for k in plain:
        assert torch.equal(never[k], plain[k])
    assert counts["predicted"] == 0
    # one that always fires sends every element of every stage to the subcell scheme untested
    pred.threshold = -1.0
    always, counts = _mood_step(op, states, bc, dt, pred, "learned")
    E = sum(bp.E for bp in op.plan.blocks)
    assert counts["predicted"] == 3 * E and counts["missed"] == 0
    for k in always:
        assert bool(torch.isfinite(always[k]).all())
