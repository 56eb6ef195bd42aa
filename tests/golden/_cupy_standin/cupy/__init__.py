"""NumPy-backed stand-in for the ``cupy`` module (fixture generation only).

TopoGPU's SolverV4 path (``src/gpu_fem/solver_v4.py``, ``multigrid_v4.py``,
``solver_v2.py``) keeps its arithmetic in CuPy calls. CuPy is not installed
in this image, so ``make_golden.py`` puts this package first on ``sys.path``
and runs the reference modules UNMODIFIED on the host. Every function maps to
the NumPy routine of the same name; arrays are a thin ``ndarray`` subclass
that adds CuPy's ``.get()``.

This is test infrastructure: nothing in the product imports it.
"""

from __future__ import annotations

import numpy as _np


class ndarray(_np.ndarray):
    """NumPy array that also answers CuPy's ``.get()``."""

    def get(self):
        return _np.asarray(self)


def _wrap(x):
    if isinstance(x, _np.ndarray) and not isinstance(x, ndarray):
        return x.view(ndarray)
    if isinstance(x, (_np.floating, _np.integer, _np.bool_)):
        return _np.asarray(x).view(ndarray)
    return x


def _wrapped(fn):
    def inner(*args, **kwargs):
        return _wrap(fn(*args, **kwargs))

    inner.__name__ = getattr(fn, "__name__", "fn")
    return inner


float16 = _np.float16
float32 = _np.float32
float64 = _np.float64
int32 = _np.int32
int64 = _np.int64
uint16 = _np.uint16
uint32 = _np.uint32
bool_ = _np.bool_


def asnumpy(x):
    return _np.asarray(x)


def asarray(x, dtype=None):
    return _wrap(_np.asarray(x, dtype=dtype).copy() if not isinstance(x, _np.ndarray) else _np.asarray(x, dtype=dtype))


def array(x, dtype=None, copy=True):
    return _wrap(_np.array(x, dtype=dtype, copy=copy))


class _AddUFunc:
    def __call__(self, *a, **k):
        return _wrap(_np.add(*a, **k))

    @staticmethod
    def at(a, idx, vals):
        _np.add.at(a, _np.asarray(idx), _np.asarray(vals))


add = _AddUFunc()


def bincount(x, weights=None, minlength=0):
    return _wrap(_np.bincount(_np.asarray(x), weights=None if weights is None else _np.asarray(weights), minlength=minlength))


class _Stream:
    def synchronize(self):
        return None


class _StreamNS:
    null = _Stream()

    @staticmethod
    def get_current_stream():
        return _Stream()

    @staticmethod
    def synchronize():
        return None


class cuda:  # noqa: N801 - mirrors cupy.cuda
    Stream = _StreamNS
    stream = _StreamNS


class _Pool:
    def free_all_blocks(self):
        return None

    def used_bytes(self):
        return 0


def get_default_memory_pool():
    return _Pool()


def get_default_pinned_memory_pool():
    return _Pool()


class _Linalg:
    norm = staticmethod(_wrapped(_np.linalg.norm))
    cholesky = staticmethod(_wrapped(_np.linalg.cholesky))
    inv = staticmethod(_wrapped(_np.linalg.inv))
    solve = staticmethod(_wrapped(_np.linalg.solve))


linalg = _Linalg()


class _RandomState:
    def __init__(self, seed=None):
        self._rs = _np.random.RandomState(seed)

    def standard_normal(self, size=None, dtype=_np.float64):
        return _wrap(self._rs.standard_normal(size).astype(dtype))


class _RandomNS:
    RandomState = _RandomState


random = _RandomNS()


def __getattr__(name):
    obj = getattr(_np, name)
    if callable(obj) and not isinstance(obj, type):
        return _wrapped(obj)
    return obj
