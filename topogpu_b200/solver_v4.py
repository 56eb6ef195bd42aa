"""``SolverV4`` with the reference's constructor and ``solve`` call.

For code that builds gpu_fem's SolverV4 directly (src/gpu_fem/solver_v4.py:
38-145 for the arguments, 147-269 for ``solve``) rather than going through
``SIMPSolver``. The arguments map onto ``StateSolver``:

* ``grid_dims`` (required), ``free``, ``F``, ``ndof``, ``KE_UNIT``;
* ``matfree_gmg_levels`` -> levels; ``gmg_fine_degree`` -> fine smoother
  degree; ``gmg_smooth_iters`` (default 2) -> coarse smoother degree;
  ``gmg_cheb_lower_frac``; ``gmg_cycle_type``; ``gmg_restart``;
* ``gmg_fine_smoother`` "fp64" / "fp32" / "bf16" -> precision "fp64" /
  "fp32" / "mixed" (here the outer Krylov vectors follow the smoother's
  precision, with an FP64 iterate and FP64 true-residual checks; the
  reference keeps an FP64 outer loop around an FP32 or BF16 smoother);
* ``gmg_smoother_type`` "chebyshev" -> the reference's Chebyshev recurrence
  (``smoother="reference"``), so FP64 runs reproduce its iterates;
* ``gmg_outer_solver`` "auto" -> PCG, or FGMRES for the BF16 smoother, as
  the reference selects (solver_v4.py:187-189);
* ``cg_tol``, ``cg_maxiter``, ``enable_warm_start``; ``enable_profiling``
  fills ``last_timing``.

``edof``, ``row_idx``, ``col_idx``, ``backend`` and the ``enable_*``
switches of the assembled and fused paths are accepted and not needed: the
operator is matrix-free on the structured grid. ``solve(rho, penal)`` takes
and returns NumPy arrays like the reference.
"""

from __future__ import annotations

import numpy as np

from .state import StateSolver

_PREC = {"fp64": "fp64", "fp32": "fp32", "bf16": "mixed"}


class SolverV4:
    def __init__(self, *args, enable_matfree_gmg: bool = True, matfree_gmg_levels: int = 4,
                 gmg_fine_smoother: str = "fp32", gmg_fine_degree: int = 2, gmg_outer_solver: str = "auto",
                 gmg_restart: int = 32, gmg_smoother_type: str = "chebyshev", gmg_cheb_lower_frac: float = 1.0 / 30.0,
                 gmg_level_precisions=None, gmg_cycle_type: str = "v", **kwargs):
        if args:
            raise TypeError("SolverV4 takes keyword arguments only")
        if not enable_matfree_gmg:
            raise ValueError("the B200 SolverV4 is the matrix-free GMG path (enable_matfree_gmg=True)")
        if gmg_fine_smoother not in _PREC:
            raise ValueError(f"gmg_fine_smoother must be one of {sorted(_PREC)}, got {gmg_fine_smoother!r}")
        if gmg_smoother_type != "chebyshev":
            raise ValueError("only gmg_smoother_type='chebyshev' is built")
        if gmg_outer_solver not in ("auto", "pcg", "fgmres"):
            raise ValueError(f"unknown gmg_outer_solver {gmg_outer_solver!r}")
        if gmg_level_precisions is not None:
            raise ValueError("per-level precisions are fixed by the precision schedule here")
        dims = kwargs.get("grid_dims")
        if dims is None:
            raise ValueError("SolverV4 requires grid_dims=(nelx, nely, nelz) for the GMG path.")
        nel = tuple(int(v) for v in dims)
        ndof = int(kwargs.get("ndof", 3 * (nel[0] + 1) * (nel[1] + 1) * (nel[2] + 1)))
        free = np.asarray(kwargs["free"], dtype=np.int64)
        F = np.asarray(kwargs["F"], dtype=np.float64)
        if F.shape != (ndof,):
            raise ValueError(f"F has {F.size} entries, expected ndof = {ndof}")
        mask = np.zeros(ndof, dtype=np.uint8)
        mask[free] = 1
        outer = gmg_outer_solver
        if outer == "auto":
            outer = "fgmres" if gmg_fine_smoother == "bf16" else "pcg"
        self.free = free
        self.ndof = ndof
        self.last_cg_iters = 0
        self.last_outer_solver = outer
        self.last_timing: dict = {}
        self._profiling = bool(kwargs.get("enable_profiling", False))
        self._state = StateSolver(
            nel, mask, F, n_levels=int(matfree_gmg_levels), precision=_PREC[gmg_fine_smoother],
            fine_degree=int(gmg_fine_degree), coarse_degree=int(kwargs.get("gmg_smooth_iters", 2)),
            cheb_lower=float(gmg_cheb_lower_frac), outer=outer, restart=int(gmg_restart),
            tol=float(kwargs.get("cg_tol", 1e-8)), maxiter=int(kwargs.get("cg_maxiter", 1000)),
            warm_start=bool(kwargs.get("enable_warm_start", False)), smoother="reference",
            cycle_type=gmg_cycle_type, KE=kwargs.get("KE_UNIT"))

    def solve(self, rho, penal: float = 3.0):
        """Compliance and dc/drho at the density rho (NumPy in, NumPy out)."""
        c, dc = self._state.solve(np.asarray(rho, dtype=np.float64), penal, timing=self._profiling)
        self.last_cg_iters = self._state.last_cg_iters
        self.last_outer_solver = self._state.last_outer_solver
        self.last_timing = dict(self._state.last_timing)
        return float(c), dc.cpu().numpy()

    def close(self):
        self._state.close()
