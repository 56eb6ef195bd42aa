"""topogpu_b200 - SolverV4 state solve and design update for NVIDIA B200.

The public names follow TopoGPU's ``topogpu`` package (src/topogpu/__init__.py)
so existing scripts switch by changing the import. All compute runs in the
hand-written CUDA library ``libtopo_b200.so`` (sm_100a); importing the
package does not load it, the first GPU call does, and a missing library is
an error (there is no CPU path).
"""

from __future__ import annotations

import importlib

__version__ = "0.1.0"

_EXPORTS = {
    "EvidenceBundle": ("topogpu_b200.evidence", "EvidenceBundle"),
    "DensityFilter": ("topogpu_b200.filter", "DensityFilter"),
    "CaseGallery": ("topogpu_b200.problem", "CaseGallery"),
    "cantilever_3d": ("topogpu_b200.problem", "cantilever_3d"),
    "side_load_cantilever": ("topogpu_b200.problem", "side_load_cantilever"),
    "benchmark_cantilever": ("topogpu_b200.problem", "benchmark_cantilever"),
    "tool_case": ("topogpu_b200.problem", "tool_case"),
    "TopologyProblem": ("topogpu_b200.problem", "TopologyProblem"),
    "ProblemSpec": ("topogpu_b200.problem_spec", "ProblemSpec"),
    "generate_bc": ("topogpu_b200.bc", "generate_bc"),
    "MatrixFreeOperator": ("topogpu_b200.operators", "MatrixFreeOperator"),
    "GMGPreconditioner": ("topogpu_b200.operators", "GMGPreconditioner"),
    "StateSolver": ("topogpu_b200.state", "StateSolver"),
    "SolverV4": ("topogpu_b200.solver_v4", "SolverV4"),
    "run_simp": ("topogpu_b200.run_simp", "run_simp"),
    "SIMPParams": ("topogpu_b200.run_simp", "SIMPParams"),
    "StepState": ("topogpu_b200.run_simp", "StepState"),
    "OCOptimizer": ("topogpu_b200.solver", "OCOptimizer"),
    "OptimizationResult": ("topogpu_b200.solver", "OptimizationResult"),
    "SIMPModel": ("topogpu_b200.solver", "SIMPModel"),
    "SIMPSolver": ("topogpu_b200.solver", "SIMPSolver"),
    "solve": ("topogpu_b200.solver", "solve"),
    "TopoContext": ("topogpu_b200.context", "TopoContext"),
}

__all__ = ["__version__", "gallery", *_EXPORTS]


def __getattr__(name: str):
    if name == "gallery":
        return importlib.import_module("topogpu_b200.problem")
    if name in _EXPORTS:
        mod, attr = _EXPORTS[name]
        return getattr(importlib.import_module(mod), attr)
    raise AttributeError(name)
