"""SciPy-backed stand-in for ``cupyx.scipy.linalg`` (fixture generation only)."""

from __future__ import annotations

import numpy as np
import scipy.linalg as _la

import cupy as _cp


def solve_triangular(a, b, trans=0, lower=False, unit_diagonal=False, overwrite_b=False, check_finite=False):
    out = _la.solve_triangular(np.asarray(a), np.asarray(b), trans=trans, lower=lower, unit_diagonal=unit_diagonal)
    return np.asarray(out).view(_cp.ndarray)
