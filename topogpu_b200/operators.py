"""Operator-level interfaces (lower drop-in boundary).

``MatrixFreeOperator`` mirrors ``MatrixFreeKff`` (src/gpu_fem/solver_v2.py:1122-1252)
and ``GMGPreconditioner`` mirrors ``GalerkinMatFreeGMG.setup/apply``
(src/gpu_fem/multigrid_v4.py:657-844), both on full-length CUDA vectors in
the reference numbering with fixed DoFs held at zero; ``pcg`` mirrors
``_cupy_pcg`` (solver_v2.py:552-624).
"""

from __future__ import annotations

import numpy as np
import torch

from .context import TopoContext


class MatrixFreeOperator:
    def __init__(self, nel, free_mask, F=None, device=None):
        self.ctx = TopoContext(nel, n_levels=1, mode="fp64")
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.free_mask = torch.as_tensor(np.asarray(free_mask, dtype=np.uint8), device=dev).contiguous()
        F = torch.zeros(self.ctx.ndof, dtype=torch.float64, device=dev) if F is None else \
            torch.as_tensor(np.asarray(F, dtype=np.float64), device=dev).contiguous()
        self.ctx.set_problem(self.free_mask, F)

    def matvec(self, u, E):
        """K(E) u; precision follows u (float64, float32 or bfloat16 input)."""
        return self.ctx.matvec(u.contiguous(), E.contiguous())

    def extract_diagonal(self, E):
        return self.ctx.diag(E.contiguous())


class GMGPreconditioner:
    """Galerkin GMG hierarchy with Chebyshev-Jacobi smoothing.

    smoother="reference" applies the reference's Chebyshev recurrence
    (multigrid_v4.py:861-889) and reproduces its V-cycle; the default
    "chebyshev" is the first-kind Chebyshev iteration with a 1.25 safety
    factor on lambda_max (the product default)."""

    def __init__(self, nel, free_mask, F=None, n_levels=4, precision="fp64", fine_degree=2, coarse_degree=2,
                 cheb_lower=1.0 / 30.0, device=None, smoother="chebyshev"):
        self.ctx = TopoContext(nel, n_levels=n_levels, mode=precision, fine_degree=fine_degree,
                               coarse_degree=coarse_degree, cheb_lower=cheb_lower, smoother=smoother)
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.free_mask = torch.as_tensor(np.asarray(free_mask, dtype=np.uint8), device=dev).contiguous()
        F = torch.zeros(self.ctx.ndof, dtype=torch.float64, device=dev) if F is None else \
            torch.as_tensor(np.asarray(F, dtype=np.float64), device=dev).contiguous()
        self.ctx.set_problem(self.free_mask, F)

    def setup(self, E):
        self.ctx.gmg_setup(E.contiguous())
        return self

    def apply(self, r):
        return self.ctx.gmg_apply(r.contiguous())

    def pcg(self, b, x0=None, tol=1e-5, maxiter=1000):
        x = torch.zeros_like(b) if x0 is None else x0.clone()
        it, rr, ok = self.ctx.pcg(b.contiguous(), x, tol, maxiter)
        return x, it, ok

    @property
    def info(self):
        return self.ctx.gmg_info()
