"""``jax.numpy`` stand-in: numpy functions returning arrays with ``.at``."""

import sys
import types

import numpy as _np


def _normalise(index, shape):
    """Expand an index to one entry per leading axis it addresses (Ellipsis/None not used here)."""
    if not isinstance(index, tuple):
        index = (index,)
    return index


def _clamped(index, shape):
    """JAX gather semantics: integer-array indices out of bounds are clamped to the edge."""
    index = _normalise(index, shape)
    out = []
    axis = 0
    for item in index:
        if item is Ellipsis:
            out.append(item)
            axis = len(shape) - (len(index) - len(out))
            continue
        if isinstance(item, _np.ndarray) and item.dtype.kind in "iu" and axis < len(shape):
            dim = shape[axis]
            item = _np.where(item < 0, item + dim, item)
            item = _np.clip(item, 0, dim - 1)
        out.append(item)
        axis += 1
    return tuple(out)


def _scatter(ufunc, array, index, value):
    """JAX scatter semantics: updates at out-of-bounds integer-array indices are dropped.
    Implemented by padding each array-indexed axis so that such updates land outside the
    cropped result."""
    index = _normalise(index, array.shape)
    pads = [0] * array.ndim
    fixed = []
    axis = 0
    for item in index:
        if isinstance(item, _np.ndarray) and item.dtype.kind in "iu" and axis < array.ndim:
            dim = array.shape[axis]
            item = _np.where(item < 0, item + dim, item)
            over = int(item.max()) - dim + 1 if item.size else 0
            pads[axis] = max(pads[axis], over)
        fixed.append(item)
        axis += 1
    if any(pads):
        padded = _np.zeros(tuple(d + p for d, p in zip(array.shape, pads)), dtype=array.dtype)
        padded[tuple(slice(0, d) for d in array.shape)] = array
        if ufunc is None:
            padded[tuple(fixed)] = value
        else:
            ufunc.at(padded, tuple(fixed), value)
        return padded[tuple(slice(0, d) for d in array.shape)].copy()
    out = _np.array(array, copy=True)
    if ufunc is None:
        out[tuple(fixed)] = value
    else:
        ufunc.at(out, tuple(fixed), value)
    return out


class _AtIndexer:
    def __init__(self, array, index):
        self.array = _np.asarray(array)
        self.index = index

    def set(self, value):
        return _wrap(_scatter(None, self.array, self.index, _np.asarray(value)))

    def add(self, value):
        return _wrap(_scatter(_np.add, self.array, self.index, _np.asarray(value)))

    def min(self, value):
        return _wrap(_scatter(_np.minimum, self.array, self.index, _np.asarray(value)))

    def max(self, value):
        return _wrap(_scatter(_np.maximum, self.array, self.index, _np.asarray(value)))


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
        index = _unwrap_index(index)
        if isinstance(index, (tuple, _np.ndarray)):
            index = _clamped(index, self.shape)
        return _wrap(_np.ndarray.__getitem__(self, index))


def _wrap(value):
    if type(value).__name__ == "Dual":
        return value
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
    if type(value).__name__ == "Dual":
        return value
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
    if type(value).__name__ == "Dual":
        return value
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
