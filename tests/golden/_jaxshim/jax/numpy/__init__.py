"""``jax.numpy`` stand-in: NumPy functions returning an ndarray subclass that
carries JAX's functional ``.at[...]`` update syntax.  Test infrastructure only.
"""
from __future__ import annotations

import types as _types

import numpy as _np


class JArray(_np.ndarray):
    """ndarray with ``x.at[idx].set/add/multiply/get`` returning copies."""

    @property
    def at(self):
        return _AtIndexer(self)


class _AtIndexer:
    def __init__(self, base):
        self._base = base

    def __getitem__(self, index):
        return _AtUpdate(self._base, index)


class _AtUpdate:
    def __init__(self, base, index):
        self._base = base
        self._index = index

    def _copy(self, value):
        dtype = _np.result_type(self._base.dtype, _np.asarray(value).dtype)
        if _np.issubdtype(self._base.dtype, _np.floating):
            dtype = self._base.dtype
        return _np.array(self._base, dtype=dtype, copy=True).view(JArray)

    def set(self, value):
        out = self._copy(value)
        out[self._index] = value
        return out

    def add(self, value):
        out = self._copy(value)
        out[self._index] += value
        return out

    def multiply(self, value):
        out = self._copy(value)
        out[self._index] *= value
        return out

    def get(self):
        return self._base[self._index]


def _j(value):
    if isinstance(value, _np.ndarray):
        return value.view(JArray) if not isinstance(value, JArray) else value
    if isinstance(value, tuple):
        return tuple(_j(v) for v in value)
    if isinstance(value, list):
        return [_j(v) for v in value]
    return value


def _wrap(fn):
    def wrapped(*args, **kwargs):
        return _j(fn(*args, **kwargs))
    wrapped.__name__ = getattr(fn, "__name__", "wrapped")
    return wrapped


def array(obj, dtype=None, copy=True, **_kwargs):
    return _np.array(obj, dtype=dtype, copy=True).view(JArray)


def asarray(obj, dtype=None, **_kwargs):
    return _np.asarray(obj, dtype=dtype).view(JArray)


ndarray = _np.ndarray
float32 = _np.float32
float64 = _np.float64
int32 = _np.int32
int64 = _np.int64
bool_ = _np.bool_
pi = _np.pi
inf = _np.inf
nan = _np.nan
dtype = _np.dtype
finfo = _np.finfo
result_type = _np.result_type
ndim = _np.ndim
newaxis = None

fft = _types.SimpleNamespace(fft=_wrap(_np.fft.fft), ifft=_wrap(_np.fft.ifft),
                             rfft=_wrap(_np.fft.rfft), irfft=_wrap(_np.fft.irfft))
linalg = _types.SimpleNamespace(norm=_wrap(_np.linalg.norm), solve=_wrap(_np.linalg.solve))


def __getattr__(name):
    target = getattr(_np, name)
    if callable(target):
        return _wrap(target)
    return target
