"""Forward-mode dual numbers for the stand-in's ``jax.jacobian``.

Covers the operations of the reference's chemistry residual (arithmetic, maximum /
minimum / clip with JAX's tie rule -- half the derivative to each side when the two
arguments are equal --, log, exp, dot with constant matrices, sum, where).
"""

import numpy as np


class Dual:
    __array_priority__ = 100

    def __init__(self, v, d):
        self.v = np.asarray(v, dtype=np.float64)
        self.d = np.asarray(d, dtype=np.float64)   # shape v.shape + (n,)

    @property
    def shape(self):
        return self.v.shape

    @property
    def ndim(self):
        return self.v.ndim

    @property
    def dtype(self):
        return self.v.dtype

    def __len__(self):
        return len(self.v)

    def __getitem__(self, idx):
        return Dual(self.v[idx], self.d[idx])


def _vd(x, n):
    if isinstance(x, Dual):
        return x.v, x.d
    x = np.asarray(x, dtype=np.float64)
    return x, np.zeros(x.shape + (n,))


def _n(*args):
    for a in args:
        if isinstance(a, Dual):
            return a.d.shape[-1]
    return 0


def _bcast(d, shape):
    return np.broadcast_to(d, shape + (d.shape[-1],))


def _maxmin(a, b, take_a, n):
    av, ad = _vd(a, n)
    bv, bd = _vd(b, n)
    v = np.where(take_a, av, bv)
    shape = v.shape
    wa = np.where(av == bv, 0.5, np.where(take_a, 1.0, 0.0))[..., None]
    return Dual(v, wa * _bcast(ad, shape) + (1.0 - wa) * _bcast(bd, shape))


def _ufunc(uf, *inputs):
    n = _n(*inputs)
    if uf is np.add:
        (av, ad), (bv, bd) = _vd(inputs[0], n), _vd(inputs[1], n)
        v = av + bv
        return Dual(v, _bcast(ad, v.shape) + _bcast(bd, v.shape))
    if uf is np.subtract:
        (av, ad), (bv, bd) = _vd(inputs[0], n), _vd(inputs[1], n)
        v = av - bv
        return Dual(v, _bcast(ad, v.shape) - _bcast(bd, v.shape))
    if uf is np.multiply:
        (av, ad), (bv, bd) = _vd(inputs[0], n), _vd(inputs[1], n)
        v = av * bv
        return Dual(v, _bcast(ad * np.asarray(bv)[..., None], v.shape) + _bcast(bd * np.asarray(av)[..., None], v.shape))
    if uf is np.true_divide:
        (av, ad), (bv, bd) = _vd(inputs[0], n), _vd(inputs[1], n)
        v = av / bv
        return Dual(v, _bcast(ad / np.asarray(bv)[..., None], v.shape)
                    - _bcast(bd * (np.asarray(av) / np.asarray(bv) ** 2)[..., None], v.shape))
    if uf is np.negative:
        av, ad = _vd(inputs[0], n)
        return Dual(-av, -ad)
    if uf is np.log:
        av, ad = _vd(inputs[0], n)
        return Dual(np.log(av), ad / av[..., None])
    if uf is np.exp:
        av, ad = _vd(inputs[0], n)
        e = np.exp(av)
        return Dual(e, ad * e[..., None])
    if uf is np.maximum:
        av, _ = _vd(inputs[0], n)
        bv, _ = _vd(inputs[1], n)
        return _maxmin(inputs[0], inputs[1], av >= bv, n)
    if uf is np.minimum:
        av, _ = _vd(inputs[0], n)
        bv, _ = _vd(inputs[1], n)
        return _maxmin(inputs[0], inputs[1], av <= bv, n)
    if uf is np.power:
        (av, ad), (bv, _) = _vd(inputs[0], n), _vd(inputs[1], n)
        v = av ** bv
        return Dual(v, _bcast(ad * (bv * av ** (bv - 1.0))[..., None], v.shape))
    if uf in (np.greater, np.greater_equal, np.less, np.less_equal, np.equal, np.isfinite):
        vals = [_vd(x, n)[0] for x in inputs]
        return uf(*vals)
    raise NotImplementedError(f"dual: ufunc {uf.__name__}")


def _function(func, args, kwargs):
    n = _n(*args)
    if func is np.dot or func is np.matmul:
        a, b = args
        if isinstance(b, Dual) and not isinstance(a, Dual):
            A = np.asarray(a)
            v = A @ b.v
            d = np.einsum("...i,in->...n", A, b.d) if A.ndim == 1 else np.einsum("ri,in->rn", A, b.d)
            return Dual(v, d)
        if isinstance(a, Dual) and not isinstance(b, Dual):
            B = np.asarray(b)
            v = a.v @ B
            return Dual(v, np.einsum("in,i...->...n", a.d, B))
        raise NotImplementedError("dual: dot of two duals")
    if func is np.sum:
        a = args[0]
        axis = kwargs.get("axis", None)
        if axis is None:
            return Dual(a.v.sum(), a.d.reshape(-1, a.d.shape[-1]).sum(axis=0))
        return Dual(a.v.sum(axis=axis), a.d.sum(axis=axis))
    if func is np.where:
        c, a, b = args
        (av, ad), (bv, bd) = _vd(a, n), _vd(b, n)
        v = np.where(c, av, bv)
        return Dual(v, np.where(np.asarray(c)[..., None], _bcast(ad, v.shape), _bcast(bd, v.shape)))
    if func is np.clip:
        a = args[0]
        lo = args[1] if len(args) > 1 else kwargs.get("a_min")
        hi = args[2] if len(args) > 2 else kwargs.get("a_max")
        return _ufunc(np.minimum, _ufunc(np.maximum, a, lo), hi)
    if func is np.abs:
        av, ad = _vd(args[0], n)
        return Dual(np.abs(av), ad * np.sign(av)[..., None])
    if func in (np.asarray, np.array):
        return args[0]
    raise NotImplementedError(f"dual: function {func.__name__}")


Dual.__array_ufunc__ = lambda self, uf, method, *inputs, **kw: _ufunc(uf, *inputs)
Dual.__array_function__ = lambda self, func, types, args, kwargs: _function(func, args, kwargs)
for _name, _uf in (("__add__", np.add), ("__sub__", np.subtract), ("__mul__", np.multiply),
                   ("__truediv__", np.true_divide), ("__pow__", np.power)):
    setattr(Dual, _name, (lambda uf: lambda self, o: _ufunc(uf, self, o))(_uf))
for _name, _uf in (("__radd__", np.add), ("__rsub__", np.subtract), ("__rmul__", np.multiply),
                   ("__rtruediv__", np.true_divide)):
    setattr(Dual, _name, (lambda uf: lambda self, o: _ufunc(uf, o, self))(_uf))
Dual.__neg__ = lambda self: _ufunc(np.negative, self)
for _name, _uf in (("__gt__", np.greater), ("__ge__", np.greater_equal), ("__lt__", np.less),
                   ("__le__", np.less_equal)):
    setattr(Dual, _name, (lambda uf: lambda self, o: _ufunc(uf, self, o))(_uf))
