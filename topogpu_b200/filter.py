"""Density filter of the public interface.

``DensityFilter(nel, radius)`` keeps the reference's host API
(src/topogpu/filter.py:10-32: dense row-normalised ``matrix()`` and
``apply()``) for small grids, and adds ``apply_cuda`` / ``apply_transpose_cuda``
which run the stencil filter of libtopo_b200.so on CUDA tensors (neighbours
at distance <= radius-1e-10, weight radius-d, rows normalised; the
``run_simp`` filter of src/gpu_fem/pub_simp_solver.py:215-243).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class DensityFilter:
    nel: tuple
    radius: float

    def matrix(self) -> np.ndarray:
        nx, ny, nz = self.nel
        i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        c = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(float)
        dist = np.sqrt(((c[:, None, :] - c[None, :, :]) ** 2).sum(axis=2))
        w = np.maximum(0.0, self.radius - dist)
        s = w.sum(axis=1)
        s[s == 0.0] = 1.0
        return w / s[:, None]

    def apply(self, rho: np.ndarray) -> np.ndarray:
        return self.matrix() @ rho

    def _ctx(self):
        from .context import TopoContext

        key = tuple(self.nel)
        cache = DensityFilter.__dict__.get("_ctx_cache")
        if cache is None:
            cache = {}
            setattr(DensityFilter, "_ctx_cache", cache)
        if key not in cache:
            cache[key] = TopoContext(key, n_levels=1, mode="fp64")
        return cache[key]

    def apply_cuda(self, rho):
        return self._ctx().filter(self.radius, rho.contiguous(), transpose=False)

    def apply_transpose_cuda(self, x):
        return self._ctx().filter(self.radius, x.contiguous(), transpose=True)
