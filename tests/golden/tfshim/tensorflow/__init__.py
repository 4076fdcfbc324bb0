"""Minimal numpy-backed stand-in for the ``tensorflow`` package.

Test infrastructure only.  TensorFlow is not installable in the build
container, so the golden-vector generator (``tests/golden/make_golden.py``)
puts this directory first on ``sys.path`` and imports the unmodified
reference modules on top of it.  Only the ~35 symbols the reference uses are
provided.  Tensors are ``numpy.ndarray`` subclasses with TF value semantics:
augmented assignment (``+=`` etc.) builds a new tensor instead of mutating in
place, as a TF EagerTensor would.

Randomness comes from one seeded ``numpy.random.Generator`` (``set_seed``),
so a generator run is reproducible; it is not TF's Philox stream.
"""
import numpy as _np
import scipy.linalg as _sla

complex128 = _np.complex128
complex64 = _np.complex64
float64 = _np.float64
float32 = _np.float32
int64 = _np.int64
int32 = _np.int32


class Tensor(_np.ndarray):
    def numpy(self):
        return _np.asarray(self).copy()

    def __iadd__(self, other):
        return _wrap(_np.add(_np.asarray(self), _np.asarray(other)))

    def __isub__(self, other):
        return _wrap(_np.subtract(_np.asarray(self), _np.asarray(other)))

    def __imul__(self, other):
        return _wrap(_np.multiply(_np.asarray(self), _np.asarray(other)))

    def __itruediv__(self, other):
        return _wrap(_np.true_divide(_np.asarray(self), _np.asarray(other)))


def _wrap(x):
    return _np.asarray(x).view(Tensor)


_rng = _np.random.default_rng(0)


def set_seed(seed):
    global _rng
    _rng = _np.random.default_rng(seed)


def function(f=None, **_kw):
    if f is None:
        return lambda g: g
    return f


def einsum(subscripts, *operands, optimize=False, **_kw):
    ops = [_np.asarray(o) for o in operands]
    return _wrap(_np.einsum(subscripts, *ops, optimize=optimize if optimize else False))


def gather(t, indices, axis=0):
    return _wrap(_np.take(_np.asarray(t), _np.asarray(indices), axis=axis))


def convert_to_tensor(x, dtype=None):
    if isinstance(x, (list, tuple)):
        x = [_np.asarray(e) if isinstance(e, _np.ndarray) else e for e in x]
    return _wrap(_np.array(x, dtype=dtype))


def constant(x, dtype=None):
    return _wrap(_np.array(x, dtype=dtype))


def complex(real, imag):
    return _wrap(_np.asarray(real) + 1j * _np.asarray(imag))


def identity(x):
    return _wrap(_np.array(x, copy=True))


def stack(values, axis=0):
    return _wrap(_np.stack([_np.asarray(v) for v in values], axis=axis))


def transpose(x, perm=None):
    return _wrap(_np.transpose(_np.asarray(x), perm))


def zeros_like(x, dtype=None):
    return _wrap(_np.zeros_like(_np.asarray(x), dtype=dtype))


def zeros(shape, dtype=float64):
    return _wrap(_np.zeros(shape, dtype=dtype))


def cast(x, dtype):
    x = _np.asarray(x)
    if _np.issubdtype(dtype, _np.complexfloating):
        return _wrap(x.astype(dtype))
    if _np.iscomplexobj(x):
        x = x.real
    return _wrap(x.astype(dtype))


def abs(x):  # noqa: A001 - TF name
    return _wrap(_np.abs(_np.asarray(x)))


def sqrt(x):
    return _wrap(_np.sqrt(_np.asarray(x)))


def reduce_sum(x, axis=None):
    return _wrap(_np.sum(_np.asarray(x), axis=axis))


def reduce_mean(x, axis=None):
    return _wrap(_np.mean(_np.asarray(x), axis=axis))


def add_n(values):
    acc = _np.asarray(values[0]).copy()
    for v in values[1:]:
        acc = acc + _np.asarray(v)
    return _wrap(acc)


def where(cond):
    return _wrap(_np.argwhere(_np.asarray(cond)))


def logical_and(a, b):
    return _wrap(_np.logical_and(a, b))


class _Math:
    conj = staticmethod(lambda x: _wrap(_np.conj(_np.asarray(x))))
    real = staticmethod(lambda x: _wrap(_np.real(_np.asarray(x))))
    abs = staticmethod(abs)
    sqrt = staticmethod(sqrt)
    add_n = staticmethod(add_n)
    accumulate_n = staticmethod(add_n)
    reduce_sum = staticmethod(reduce_sum)


math = _Math()


class _DTypes:
    cast = staticmethod(cast)


dtypes = _DTypes()


class _Random:
    @staticmethod
    def normal(shape, mean=0.0, stddev=1.0, dtype=float64, **_kw):
        return _wrap(_rng.normal(mean, stddev, size=shape).astype(dtype))

    @staticmethod
    def uniform(shape, minval=0, maxval=None, dtype=float64, **_kw):
        if maxval is None:
            maxval = 1
        if _np.issubdtype(dtype, _np.integer):
            return _wrap(_rng.integers(minval, maxval, size=shape).astype(dtype))
        return _wrap(_rng.uniform(minval, maxval, size=shape).astype(dtype))


random = _Random()


def _batched_sqrtm(a):
    a = _np.ascontiguousarray(a)
    out = _np.empty(a.shape, dtype=_np.complex128)
    flat_in = a.reshape(-1, a.shape[-2], a.shape[-1])
    flat_out = out.reshape(-1, a.shape[-2], a.shape[-1])
    for i in range(flat_in.shape[0]):
        flat_out[i] = _sla.sqrtm(flat_in[i])
    return out


class _Linalg:
    expm = staticmethod(lambda x: _wrap(_sla.expm(_np.asarray(x))))
    sqrtm = staticmethod(lambda x: _wrap(_batched_sqrtm(x)))
    inv = staticmethod(lambda x: _wrap(_np.linalg.inv(_np.asarray(x))))
    det = staticmethod(lambda x: _wrap(_np.linalg.det(_np.asarray(x))))

    @staticmethod
    def qr(x):
        q, r = _np.linalg.qr(_np.asarray(x))
        return _wrap(q), _wrap(r)


linalg = _Linalg()


class _Threading:
    @staticmethod
    def set_intra_op_parallelism_threads(_n):
        pass

    @staticmethod
    def set_inter_op_parallelism_threads(_n):
        pass


class _Config:
    threading = _Threading()


config = _Config()
