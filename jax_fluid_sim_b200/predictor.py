"""Learned troubled-cell predictor for the MOOD subcell fallback.

No reference counterpart: the reference only has the a-posteriori detector
(``hybrid/limiter.py:150-185,285-300``).  The predictor reads a stage's base state and
flags the elements that the detector is expected to reject; inside
``HybridSSPRK3.checked_step`` those go to the subcell finite-volume scheme without the
failed high-order attempt, while every other element is still tested a posteriori, so
the detector stays the fallback and the arbiter.

Everything runs in hand-written kernels (``csrc/mlp_kernels.cuh``): features
(``dgb_mlp_features``), training (``dgb_mlp_train_step``: forward, backward, Adam on float32
master weights) and inference (``dgb_mlp_infer``: float16 weights, float32 accumulation).
"""

import ctypes

import numpy as np
import torch

from . import _native as N
from .operators import _stream_ptr

FEATURES, HIDDEN, PARAMS = 8, 64, 8961
MODES = {"off": 0, "learned": 1, "evaluate": 2}


def _lib():
    L = N.lib()
    if not getattr(L, "_mlp_bound", False):
        vp, i64, f = ctypes.c_void_p, ctypes.c_int64, ctypes.c_float
        sig = {
            "dgb_mlp_features": [vp, ctypes.POINTER(N.State), vp, vp],
            "dgb_mlp_infer": [vp, vp, vp, i64, f, vp, vp, vp],
            "dgb_mlp_train_step": [vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int, f, f, ctypes.c_int, vp, vp],
            "dgb_plan_set_predictor": [vp, vp, vp, f, ctypes.c_int],
            "dgb_plan_predictor_counts": [vp, ctypes.POINTER(ctypes.c_int64), ctypes.c_int],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L._mlp_bound = True
    return L


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class TroubledCellPredictor:
    """8 -> 64 -> 64 -> 64 -> 1 MLP on per-element features of a stage's base state."""

    def __init__(self, operator, threshold=0.5, seed=0):
        self.operator = operator
        self.threshold = float(threshold)
        g = torch.Generator().manual_seed(seed)
        w = torch.zeros(PARAMS)
        off = 0
        for fan_in, fan_out in ((FEATURES, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, 1)):
            n = fan_in * fan_out
            w[off:off + n] = torch.randn(n, generator=g) * (2.0 / fan_in) ** 0.5     # He initialisation
            off += n + fan_out                                                        # biases start at 0
        self.weights = w.cuda()
        self.grad = torch.zeros_like(self.weights)
        self.m = torch.zeros_like(self.weights)
        self.v = torch.zeros_like(self.weights)
        self.weights16 = self.weights.half()
        self.norm = torch.cat([torch.zeros(FEATURES), torch.ones(FEATURES)]).cuda()
        self.steps = 0

    # ---------------------------------------------------------------- data
    def features(self, states):
        """(sum of E, 8) float32 features of ``states`` in block order."""
        op = self.operator
        U = op.to_device(states)
        total = sum(bp.E for bp in op.plan.blocks)
        out = torch.empty((total, FEATURES), dtype=torch.float32, device="cuda")
        st = op.native.state(op._blocks(U))
        N.check(_lib().dgb_mlp_features(op.native.handle, ctypes.byref(st), _ptr(out), _stream_ptr()))
        return out

    def labelled_samples(self, states, dt, boundary_state, limiter):
        """Features of ``states`` and the detector's flags on its first SSP-RK stage (the
        unlimited forward-Euler candidate), the pair the predictor learns."""
        op = self.operator
        U = op.to_device(states)
        R = op.rhs(U, boundary_state)
        cand = {k: U[k] + dt * R[k] for k in U}
        flags = limiter.troubled(cand)
        y = torch.cat([flags[k].reshape(-1).to(torch.uint8) for k in op.names])
        return self.features(U), y

    # ---------------------------------------------------------------- training
    def fit(self, X, y, epochs=20, batch=4096, lr=2e-3, pos_weight=None, seed=0):
        """Adam on weighted binary cross-entropy; returns the loss of every epoch."""
        X = X.contiguous().float().cuda()
        y = y.contiguous().to(torch.uint8).cuda()
        n = X.shape[0]
        mean = X.mean(0)
        std = X.std(0).clamp_min(1e-6)
        self.norm.copy_(torch.cat([mean, 1.0 / std]))      # in place: an attached plan keeps the pointer
        pos = int(y.sum().item())
        if pos_weight is None:
            pos_weight = float(min(max((n - pos) / max(pos, 1), 1.0), 1000.0))
        g = torch.Generator(device="cuda").manual_seed(seed)
        loss = torch.zeros(1, device="cuda")
        history = []
        L = _lib()
        for _ in range(epochs):
            order = torch.randperm(n, generator=g, device="cuda").to(torch.int32)
            loss.zero_()
            for s in range(0, n, batch):
                idx = order[s:s + batch]
                self.steps += 1
                N.check(L.dgb_mlp_train_step(_ptr(self.weights), _ptr(self.grad), _ptr(self.m), _ptr(self.v),
                                             _ptr(self.weights16), _ptr(self.norm), _ptr(X), _ptr(y), _ptr(idx),
                                             int(idx.numel()), float(pos_weight), float(lr), self.steps,
                                             _ptr(loss), _stream_ptr()))
            history.append(float(loss.item()) * batch / n)
        return history

    def predict(self, X):
        X = X.contiguous().float().cuda()
        prob = torch.empty(X.shape[0], dtype=torch.float32, device="cuda")
        N.check(_lib().dgb_mlp_infer(_ptr(self.weights16), _ptr(self.norm), _ptr(X), X.shape[0], self.threshold,
                                     _ptr(prob), None, _stream_ptr()))
        return prob

    # ---------------------------------------------------------------- use inside the step
    def attach(self, mode="learned"):
        """Run inside the MOOD stages of the operator's checked step (``mode`` learned or
        evaluate; "off" detaches)."""
        op = self.operator
        N.check(_lib().dgb_plan_set_predictor(op.native.handle, _ptr(self.weights16), _ptr(self.norm),
                                              self.threshold, MODES[mode]))

    def counts(self, reset=True):
        out = (ctypes.c_int64 * 5)()
        N.check(_lib().dgb_plan_predictor_counts(self.operator.native.handle, out, int(reset)))
        return {"predicted": out[1], "missed": out[2], "false_positive": out[3], "hit": out[4]}


def confusion(pred, truth):
    """Missed-cell and false-positive rates of boolean predictions against detector flags."""
    pred = np.asarray(pred, bool)
    truth = np.asarray(truth, bool)
    pos, neg = truth.sum(), (~truth).sum()
    return {"missed_rate": float((truth & ~pred).sum() / max(pos, 1)),
            "false_positive_rate": float((pred & ~truth).sum() / max(neg, 1)),
            "positives": int(pos), "samples": int(truth.size)}
