"""``jax.lax`` stand-in: control flow executed eagerly in Python."""

import types

import numpy as _np

from .numpy import _wrap


Precision = types.SimpleNamespace(HIGHEST="highest", HIGH="high", DEFAULT="default")


def cond(predicate, true_function, false_function, *operands):
    if bool(_np.asarray(predicate)):
        return true_function(*operands)
    return false_function(*operands)


def fori_loop(lower, upper, body, init):
    value = init
    for i in range(int(lower), int(upper)):
        value = body(i, value)
    return value


def while_loop(condition, body, init):
    value = init
    while bool(_np.asarray(condition(value))):
        value = body(value)
    return value


def scan(function, init, xs, length=None):
    carry = init
    outputs = []
    count = length if xs is None else len(xs)
    for i in range(count):
        carry, y = function(carry, None if xs is None else xs[i])
        outputs.append(y)
    if outputs and outputs[0] is not None:
        stacked = _wrap(_np.stack([_np.asarray(o) for o in outputs]))
    else:
        stacked = None
    return carry, stacked
