"""What the learned troubled-cell predictor buys in the checked MOOD step, on the benchmark's
sphere grid (smallest size, 416 P3 hexahedra) from its shocked start.

1. Skipping is exact.  When every element is predicted troubled (threshold below 0) the
   learned step sends them all to the subcell scheme without their high-order update and
   without the a-posteriori test; the plain step with a detector that flags every element
   (sensor threshold below 0) recomputes the same elements after computing that update.  The
   subcell scheme uses only the base state and the viscous residual of a troubled element
   (formed for the flagged elements by the same kernel in both steps), so the two steps must
   agree bit for bit.
2. The trained network gains.  Trained on ten plain steps, in evaluate mode (the plain step,
   every element still tested) it predicts at least half of the detector's flags, i.e. those
   elements' failed high-order attempts are the ones the learned step skips; the learned step
   stays admissible, the elements it missed are caught by the detector (counted), and its
   density stays within 5e-2 (relative L2) of the plain step's: its false positives get the
   subcell update, which is not the high-order one."""

import numpy as np
import pytest
import torch

from jax_fluid_sim_b200 import workloads

pytestmark = pytest.mark.gpu


def _setup(sensor_threshold=5e-2):
    import jax_fluid_sim_b200 as jfs
    solver, op, bc, U = workloads.sphere_case("tiny", 3, "float64")
    lim = jfs.HybridMOODSubcellLimiter(op, threshold=sensor_threshold, positivity=jfs.HybridPositivityLimiter(op))
    integ = jfs.HybridSSPRK3(op, cfl=0.3, limiter=lim)
    return op, bc, U, lim, integ


def test_skipping_the_high_order_attempt_is_exact():
    from jax_fluid_sim_b200.predictor import TroubledCellPredictor
    op, bc, U, lim, integ = _setup(sensor_threshold=-1.0)
    dt = integ.stable_dt(U, bc)
    plain = {k: v.clone() for k, v in U.items()}
    integ.checked_step_inplace(plain, dt, bc)
    pred = TroubledCellPredictor(op, threshold=-1.0)      # every element predicted
    pred.attach("learned")
    pred.counts(reset=True)
    learned = {k: v.clone() for k, v in U.items()}
    status = integ.checked_step_inplace(learned, dt, bc)
    counts = pred.counts(reset=True)
    pred.attach("off")
    E = sum(bp.E for bp in op.plan.blocks)
    assert counts["predicted"] == 3 * E                   # every element, every stage
    assert bool(status.view(torch.int32)[0].item())
    for k in U:
        assert torch.equal(learned[k], plain[k])


def test_trained_predictor_skips_most_failed_attempts():
    from jax_fluid_sim_b200.predictor import TroubledCellPredictor
    op, bc, U, lim, integ = _setup()
    dt = integ.stable_dt(U, bc)
    pred = TroubledCellPredictor(op, threshold=0.5, seed=0)
    Xs, ys = [], []
    cur = {k: v.clone() for k, v in U.items()}
    for _ in range(10):
        X, y = pred.labelled_samples(cur, dt, bc, lim)
        Xs.append(X)
        ys.append(y)
        integ.checked_step_inplace(cur, dt, bc)
    X, y = torch.cat(Xs), torch.cat(ys)
    assert int(y.sum().item()) > 0
    pred.fit(X, y, epochs=60, batch=1024)
    pred.attach("evaluate")
    pred.counts(reset=True)
    ev = {k: v.clone() for k, v in cur.items()}
    integ.checked_step_inplace(ev, dt, bc)
    c = pred.counts(reset=True)
    flagged = c["hit"] + c["missed"]
    assert flagged > 0
    recall = c["hit"] / flagged
    assert recall >= 0.5, c
    pred.attach("learned")
    pred.counts(reset=True)
    learned = {k: v.clone() for k, v in cur.items()}
    status = integ.checked_step_inplace(learned, dt, bc)
    lc = pred.counts(reset=True)
    pred.attach("off")
    assert bool(status.view(torch.int32)[0].item())
    assert lc["predicted"] >= c["hit"] // 2               # the skipped attempts of the learned step
    plain = {k: v.clone() for k, v in cur.items()}
    integ.checked_step_inplace(plain, dt, bc)
    num = sum(float(((learned[k][..., 0] - plain[k][..., 0]) ** 2).sum()) for k in plain)
    den = sum(float((plain[k][..., 0] ** 2).sum()) for k in plain)
    l2 = (num / den) ** 0.5
    # the false positives' subcell update moves the solution: bounded, not zero
    assert np.isfinite(l2) and l2 < 5e-2, l2
