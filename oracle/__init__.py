"""CPU oracle for the SolverV4 state solve and design update (TEST INFRASTRUCTURE).

This package restates TopoGPU's SolverV4 hot path in NumPy/SciPy so that the
CUDA path can be checked against it. It is the checker, never the product:
only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import it. ``topogpu_b200`` never imports it and has no CPU fallback.

Parity is pinned: ``tests/golden/make_golden.py`` runs the UNMODIFIED
reference (``src/gpu_fem/*.py``, ``src/topogpu/*.py``) on a NumPy-backed
``cupy`` stand-in and stores its outputs as ``tests/golden/*.npz``;
``tests/test_oracle_golden.py`` checks every function here against them.

Modules
-------
fem      hex8 stiffness, element->DoF map, boundary conditions, K.u, diag,
         element-energy sensitivity            (pub_simp_solver.py, solver_v2.py,
                                                bc_generator.py, solver_v4.py)
gmg      prolongation, injection free sets, level-1 Galerkin, R.A.P, Chebyshev,
         V-cycle, coarsest solve               (solver_v2.py, multigrid_v4.py)
krylov   PCG and FGMRES                        (solver_v2.py, multigrid_v4.py)
design   OC updates and the density filter     (topogpu/solver.py,
                                                pub_simp_solver.py, topogpu/filter.py)
simp     SolverV4-equivalent state solve and SIMP loops
"""
