"""Minimal numpy-backed stand-in for the JAX surface the reference's hybrid
solver uses, so that the reference's own Python can run in a container without
JAX to produce golden fixtures.

Only the fixture generator in ``tests/golden/make_golden.py`` puts this on
``sys.path``.  Semantics covered: immutable-style ``.at[...]`` updates (copy
then ``np.add.at``/``np.minimum.at``), ``jit``/``vmap``/``jacobian``,
``lax.cond/fori_loop/scan/while_loop``, ``tree.map``, ``config``.
``jacobian`` is forward-mode differentiation with dual numbers (``_dual.py``),
following JAX's derivative conventions for ``maximum``/``minimum``/``clip``.
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
    """Forward-mode derivative with JAX's tie rule for max/min/clip (see _dual.py)."""
    from ._dual import Dual

    def jac(x):
        x = _np.asarray(x, dtype=_np.float64)
        n = x.size
        seed = Dual(x, _np.eye(n).reshape(x.shape + (n,)))
        out = function(seed)
        return _wrap(_np.asarray(out.d).reshape(out.v.shape + x.shape))

    return jac
