"""``jax.numpy`` stand-in: numpy functions returning arrays with ``.at``."""

import sys
import types

import numpy as _np


class _AtIndexer:
    def __init__(self, array, index):
        self.array = array
        self.index = index

    def set(self, value):
        out = _np.array(self.array, copy=True)
        out[self.index] = _np.asarray(value)
        return _wrap(out)

    def add(self, value):
        out = _np.array(self.array, copy=True)
        _np.add.at(out, self.index, _np.asarray(value))
        return _wrap(out)

    def min(self, value):
        out = _np.array(self.array, copy=True)
        _np.minimum.at(out, self.index, _np.asarray(value))
        return _wrap(out)

    def max(self, value):
        out = _np.array(self.array, copy=True)
        _np.maximum.at(out, self.index, _np.asarray(value))
        return _wrap(out)


class _At:
    def __init__(self, array):
        self.array = array

    def __getitem__(self, index):
        index = _unwrap_index(index)
        return _AtIndexer(self.array, index)


def _unwrap_index(index):
    if isinstance(index, tuple):
        return tuple(_unwrap_index(i) for i in index)
    if isinstance(index, JArray):
        return _np.asarray(index)
    return index


class JArray(_np.ndarray):
    @property
    def at(self):
        return _At(self)

    def __getitem__(self, index):
        return _wrap(_np.ndarray.__getitem__(self, _unwrap_index(index)))


def _wrap(value):
    if isinstance(value, _np.ndarray) and not isinstance(value, JArray):
        return value.view(JArray)
    if isinstance(value, (_np.floating, _np.integer, _np.bool_)):
        return _np.asarray(value).view(JArray)
    if isinstance(value, tuple):
        return tuple(_wrap(v) for v in value)
    if isinstance(value, list):
        return [_wrap(v) for v in value]
    return value


def _plain(value):
    if isinstance(value, JArray):
        return _np.asarray(value)
    if isinstance(value, (list, tuple)):
        return type(value)(_plain(v) for v in value)
    return value


def _wrapped(function):
    def call(*args, **kwargs):
        kwargs.pop("precision", None)
        return _wrap(function(*[_plain(a) for a in args], **{k: _plain(v) for k, v in kwargs.items()}))

    call.__name__ = getattr(function, "__name__", "f")
    return call


def einsum(subscripts, *operands, **kwargs):
    kwargs.pop("precision", None)
    ops = [_np.asarray(o) for o in operands]
    if len(ops) > 2:
        return _wrap(_np.einsum(subscripts, *ops, optimize=True))
    return _wrap(_np.einsum(subscripts, *ops))


def asarray(value, dtype=None):
    if isinstance(value, (list, tuple)):
        value = [_np.asarray(v) if isinstance(v, JArray) else v for v in value]
    return _wrap(_np.asarray(value, dtype=dtype))


array = asarray

_PASSTHROUGH = {
    "float64": _np.float64, "float32": _np.float32, "int32": _np.int32,
    "int64": _np.int64, "bool_": _np.bool_, "pi": _np.pi, "inf": _np.inf,
    "nan": _np.nan, "finfo": _np.finfo, "ndarray": JArray, "newaxis": None,
}


def _module_getattr(name):
    if name in _PASSTHROUGH:
        return _PASSTHROUGH[name]
    target = getattr(_np, name)
    if callable(target) and not isinstance(target, type):
        return _wrapped(target)
    return target


linalg = types.ModuleType("jax.numpy.linalg")
for _name in ("inv", "det", "solve", "pinv", "norm", "eigvalsh", "eigh", "cholesky"):
    setattr(linalg, _name, _wrapped(getattr(_np.linalg, _name)))

_this = sys.modules[__name__]


def __getattr__(name):
    return _module_getattr(name)


sys.modules.setdefault("jax.numpy.linalg", linalg)
