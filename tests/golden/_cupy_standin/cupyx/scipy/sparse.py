"""SciPy-backed stand-in for ``cupyx.scipy.sparse`` (fixture generation only).

``csr_matrix`` subclasses SciPy's CSR matrix so that products, transposes and
dtype casts return the wrapped ``cupy.ndarray`` / ``csr_matrix`` types the
reference code expects.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as _sp

import cupy as _cp


class csr_matrix(_sp.csr_matrix):  # noqa: N801 - mirrors cupyx name
    def __init__(self, arg1, shape=None, dtype=None, copy=False):
        if isinstance(arg1, tuple):
            arg1 = tuple(np.asarray(a) if isinstance(a, np.ndarray) else a for a in arg1)
        super().__init__(arg1, shape=shape, dtype=dtype, copy=copy)

    def _wrapout(self, out):
        if isinstance(out, _sp.spmatrix) or isinstance(out, _sp.sparray):
            return csr_matrix(out.tocsr())
        if isinstance(out, np.ndarray):
            return out.view(_cp.ndarray)
        return out

    def __matmul__(self, other):
        if isinstance(other, np.ndarray):
            return _sp.csr_matrix.__matmul__(self, np.asarray(other)).view(_cp.ndarray)
        return self._wrapout(_sp.csr_matrix.__matmul__(self, other))

    def dot(self, other):
        return self.__matmul__(other)

    @property
    def T(self):
        return csr_matrix(_sp.csr_matrix(self).T.tocsr())

    def tocsr(self, copy=False):
        return csr_matrix(_sp.csr_matrix(self), copy=copy)

    def astype(self, dtype, casting="unsafe", copy=True):
        return csr_matrix(_sp.csr_matrix(self).astype(dtype))

    def diagonal(self, k=0):
        return np.asarray(_sp.csr_matrix(self).diagonal(k)).view(_cp.ndarray)

    def toarray(self, order=None, out=None):
        return np.asarray(_sp.csr_matrix(self).toarray()).view(_cp.ndarray)
