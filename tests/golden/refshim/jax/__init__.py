"""Minimal numpy-backed stand-in for the JAX surface the reference's hybrid
solver uses, so that the reference's own Python can run in a container without
JAX to produce golden fixtures.

Only the fixture generator in ``tests/golden/make_golden.py`` puts this on
``sys.path``.  Semantics covered: immutable-style ``.at[...]`` updates (copy
then ``np.add.at``/``np.minimum.at``), ``jit``/``vmap``/``jacobian``,
``lax.cond/fori_loop/scan/while_loop``, ``tree.map``, ``config``.
``jacobian`` is a central finite difference; the reference only uses it inside
a Newton iteration whose converged root does not depend on it.
"""

import types

import numpy as _np

from . import numpy  # noqa: F401  (registers jax.numpy)
from .numpy import JArray, _wrap
from . import lax  # noqa: F401


Array = JArray


class _Config:
    x64_enabled = True

    def update(self, name, value):
        if name == "jax_enable_x64" and not value:
            raise RuntimeError("the stand-in runs in float64 only")


config = _Config()


def jit(function=None, **kwargs):
    if function is None:
        return lambda f: f
    return function


def _tree_leaves_map(function, tree, *rest):
    if isinstance(tree, dict):
        return {k: _tree_leaves_map(function, tree[k], *[r[k] for r in rest]) for k in tree}
    if isinstance(tree, (tuple, list)):
        out = [_tree_leaves_map(function, t, *[r[i] for r in rest]) for i, t in enumerate(tree)]
        return type(tree)(out)
    return function(tree, *rest)


tree = types.SimpleNamespace(map=_tree_leaves_map)


def _stack_results(results):
    first = results[0]
    if isinstance(first, dict):
        return {k: _stack_results([r[k] for r in results]) for k in first}
    if isinstance(first, tuple):
        return tuple(_stack_results([r[i] for r in results]) for i in range(len(first)))
    return _wrap(_np.stack([_np.asarray(r) for r in results], axis=0))


def vmap(function, in_axes=0, out_axes=0):
    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        size = None
        for a, ax in zip(args, axes):
            if ax is not None:
                size = _np.asarray(a).shape[ax]
                break
        results = []
        for i in range(size):
            call = []
            for a, ax in zip(args, axes):
                if ax is None:
                    call.append(a)
                else:
                    call.append(_wrap(_np.take(_np.asarray(a), i, axis=ax)))
            results.append(function(*call))
        return _stack_results(results)

    return mapped


def jacobian(function):
    def jac(x):
        x = _np.asarray(x, dtype=_np.float64)
        f0 = _np.asarray(function(_wrap(x.copy())))
        out = _np.zeros(f0.shape + x.shape)
        flat = x.reshape(-1)
        for j in range(flat.size):
            h = 1.0e-6 * max(abs(flat[j]), 1.0e-12)
            xp = flat.copy()
            xm = flat.copy()
            xp[j] += h
            xm[j] -= h
            fp = _np.asarray(function(_wrap(xp.reshape(x.shape))))
            fm = _np.asarray(function(_wrap(xm.reshape(x.shape))))
            out.reshape(f0.shape + (-1,))[..., j] = (fp - fm) / (2.0 * h)
        return _wrap(out)

    return jac
