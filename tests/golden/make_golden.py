"""Generate golden fixtures by running the UNMODIFIED TopoGPU reference.

Run in the build container (where the reference source is mounted):

    python tests/golden/make_golden.py /path/to/TopoGPU

The reference's CuPy calls are served by the NumPy-backed stand-in in
``tests/golden/_cupy_standin`` (CuPy itself is not installed). Outputs are
small ``.npz`` files next to this script; the GPU box never needs the
reference. Every array is produced by reference code paths:

  ke_edof.npz      KE_UNIT_3D, _edof_table_3d            (pub_simp_solver.py:157-207)
  bc.npz           generate_bc on gallery cantilevers    (bc_generator.py:381-447)
  matvec.npz       MatrixFreeKff.matvec / extract_diagonal (solver_v2.py:1183-1252)
  transfer.npz     _build_scalar_prolongation, _coarse_free_dofs_injection
  galerkin.npz     GalerkinMatFreeGMG.setup: K1 (level-1 Galerkin), K2, K3 (R.A.P),
                   lambda estimates, one V-cycle apply    (multigrid_v4.py)
  krylov.npz       _cupy_pcg and _cupy_fgmres with the GMG preconditioner
  solverv4.npz     SolverV4 + topogpu._oc_update, 3 SIMP iterations, 24x12x6
                   cantilever (FP64 and FP32 smoothers)
  oc.npz           topogpu.solver._oc_update on seeded inputs
  filter.npz       _build_density_filter (rmin 1.5, 2.0), DensityFilter.matrix
  run_simp.npz     run_simp on the 24x12x6 cantilever (rmin 1.5, move 0.2, no Heaviside)
  run_simp_heaviside.npz  run_simp on the same mesh with Heaviside
                   projection at beta 1 (the SIMPParams default) and beta 8
  wcycle.npz       GalerkinMatFreeGMG(cycle_type="w").apply and PCG on the
                   galerkin.npz hierarchies
  run_simp_control.npz  run_simp on its 3-D tip-load cantilever preset with
                   a scripted controller (initial action, beta/penal/move
                   changes, a restart from the best design, a stop, a tail)
  run_simp_resume.npz  run_simp on the 3-D preset interrupted after 4 of 7
                   iterations (checkpoint_every 2) and resumed: both legs
  ckpt_24x12x6_cantilever.{npz,json}  the checkpoint run_simp writes after
                   iteration 2 of that 24x12x6 run (checkpoint_every 1)

``python make_golden.py [REF_ROOT] [--only heaviside|checkpoint|wcycle|control|resume]``
regenerates all fixtures, or only the named group.
"""

from __future__ import annotations

import io
import sys
from contextlib import redirect_stdout
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _setup(ref_root: Path) -> None:
    sys.path.insert(0, str(HERE / "_cupy_standin"))
    sys.path.insert(0, str(ref_root / "src"))
    sys.path.insert(0, str(ref_root))


def _csr(prefix: str, M) -> dict:
    M = M.tocsr()
    M.sort_indices()
    return {f"{prefix}_indptr": M.indptr.astype(np.int64), f"{prefix}_indices": M.indices.astype(np.int64),
            f"{prefix}_data": np.asarray(M.data, dtype=np.float64), f"{prefix}_shape": np.array(M.shape)}


def cantilever_bc(nel):
    nelx, nely, nelz = nel
    nny, nnz = nely + 1, nelz + 1
    ndof = 3 * (nelx + 1) * nny * nnz
    face = np.arange(nny * nnz)
    fixed = np.sort(np.concatenate([3 * face, 3 * face + 1, 3 * face + 2]))
    free = np.setdiff1d(np.arange(ndof), fixed)
    F = np.zeros(ndof)
    edge = nelx * nny * nnz + np.arange(nny) * nnz
    F[3 * edge + 2] = -1.0 / len(edge)
    return fixed, free, F, ndof


def main(ref_root: str) -> None:
    _setup(Path(ref_root))
    import gpu_fem.multigrid_v4 as mg
    import gpu_fem.solver_v2 as sv2
    from gpu_fem.bc_generator import generate_bc
    from gpu_fem.pub_simp_solver import (KE_UNIT_3D, SIMPParams, _build_density_filter,
                                         _edof_table_3d, run_simp)
    from gpu_fem.solver_v4 import SolverV4
    import topogpu as tg
    from topogpu.solver import _oc_update

    import cupy as cp

    out = {}
    # ---- KE / edof ------------------------------------------------------
    np.savez_compressed(HERE / "ke_edof.npz", KE=KE_UNIT_3D, edof_432=_edof_table_3d(4, 3, 2),
                        edof_753=_edof_table_3d(7, 5, 3))

    # ---- BCs from the public gallery -----------------------------------
    d = {}
    for nel in [(4, 3, 2), (24, 12, 6), (7, 5, 3)]:
        p = tg.gallery.cantilever_3d(nel=nel, volfrac=0.3)
        bc = generate_bc(p.spec)
        tag = "x".join(map(str, nel))
        d[f"free_{tag}"] = bc.free_dofs.astype(np.int64)
        d[f"F_{tag}"] = bc.F
        p2 = tg.gallery.side_load_cantilever(nel=nel)
        bc2 = generate_bc(p2.spec)
        d[f"side_free_{tag}"] = bc2.free_dofs.astype(np.int64)
        d[f"side_F_{tag}"] = bc2.F
    np.savez_compressed(HERE / "bc.npz", **d)

    # ---- matvec / diagonal ---------------------------------------------
    d = {}
    for nel in [(24, 12, 6), (7, 5, 3)]:
        tag = "x".join(map(str, nel))
        edof = _edof_table_3d(*nel)
        fixed, free, F, ndof = cantilever_bc(nel)
        rng = np.random.default_rng(7)
        rho = rng.uniform(0.001, 1.0, edof.shape[0])
        E = 1e-9 + (1 - 1e-9) * rho**3
        u = rng.standard_normal(len(free))
        op = sv2.MatrixFreeKff(cp.asarray(edof), cp.asarray(KE_UNIT_3D), cp.asarray(free.astype(np.int32)),
                               len(free), ndof)
        d[f"rho_{tag}"] = rho
        d[f"u_{tag}"] = u
        d[f"y64_{tag}"] = np.asarray(op.matvec(cp.asarray(u), cp.asarray(E)))
        d[f"y32_{tag}"] = np.asarray(op.matvec(cp.asarray(u.astype(np.float32)), cp.asarray(E.astype(np.float32))))
        d[f"diag_{tag}"] = np.asarray(op.extract_diagonal(cp.asarray(E)))
    np.savez_compressed(HERE / "matvec.npz", **d)

    # ---- transfers ------------------------------------------------------
    d = {}
    pairs = [((24, 12, 6), (12, 6, 3)), ((12, 6, 3), (6, 3, 1)), ((6, 3, 1), (3, 1, 1)),
             ((7, 5, 3), (3, 2, 1)), ((3, 2, 1), (1, 1, 1)), ((1, 1, 1), (1, 1, 1))]
    for fine, coarse in pairs:
        tag = "x".join(map(str, fine)) + "_" + "x".join(map(str, coarse))
        d.update(_csr(f"P_{tag}", sv2._build_scalar_prolongation(*fine, *coarse)))
        fixed, free, F, ndof = cantilever_bc(fine)
        d[f"inj_{tag}"] = sv2._coarse_free_dofs_injection(*fine, *coarse, free).astype(np.int64)
    np.savez_compressed(HERE / "transfer.npz", **d)

    # ---- GMG setup / apply ---------------------------------------------
    d = {}
    for nel, nlev in [((24, 12, 6), 4), ((7, 5, 3), 3)]:
        tag = "x".join(map(str, nel))
        edof = _edof_table_3d(*nel)
        fixed, free, F, ndof = cantilever_bc(nel)
        rng = np.random.default_rng(11)
        rho = rng.uniform(0.05, 1.0, edof.shape[0])
        E = 1e-9 + (1 - 1e-9) * rho**3
        free_gpu = cp.asarray(free.astype(np.int32))
        op = sv2.MatrixFreeKff(cp.asarray(edof), cp.asarray(KE_UNIT_3D), free_gpu, len(free), ndof)
        with redirect_stdout(io.StringIO()):
            g = mg.GalerkinMatFreeGMG(mf_op=op, free=free.astype(np.int32), free_gpu=free_gpu, nelx=nel[0],
                                      nely=nel[1], nelz=nel[2], KE_UNIT=KE_UNIT_3D, n_levels=nlev,
                                      fine_smoother="fp64", fine_smoother_degree=2)
            g.setup(cp.asarray(E))
        d[f"rho_{tag}"] = rho
        for lv in range(1, nlev):
            d.update(_csr(f"K{lv}_{tag}", g._K_gpu[lv]))
            d[f"free{lv}_{tag}"] = np.asarray(g._free_per_level[lv]).astype(np.int64)
        d[f"lam_{tag}"] = np.array(g._lambda_max_per_level)
        r = rng.standard_normal(len(free))
        d[f"r_{tag}"] = r
        d[f"z_{tag}"] = np.asarray(g.apply(cp.asarray(r)))
        d[f"chol_mode_{tag}"] = np.array(g._coarse_chol_mode)
        # krylov on this hierarchy
        Fd = cp.asarray(F[free])
        x, it, ok = sv2._cupy_pcg(lambda v: op.matvec(v, cp.asarray(E)), Fd, g.apply, tol=1e-8, maxiter=500)
        d[f"pcg_x_{tag}"] = np.asarray(x)
        d[f"pcg_it_{tag}"] = np.array(it)
        x2, it2, ok2 = mg._cupy_fgmres(lambda v: op.matvec(v, cp.asarray(E)), Fd, g.apply, tol=1e-8,
                                       maxiter=500, restart=32)
        d[f"fgmres_x_{tag}"] = np.asarray(x2)
        d[f"fgmres_it_{tag}"] = np.array(it2)
    np.savez_compressed(HERE / "galerkin.npz", **d)

    # ---- SolverV4 + OC, 24x12x6 cantilever --------------------------------
    d = {}
    nel = (24, 12, 6)
    edof = _edof_table_3d(*nel)
    fixed, free, F, ndof = cantilever_bc(nel)
    for prec in ["fp64", "fp32"]:
        with redirect_stdout(io.StringIO()):
            s = SolverV4(edof=edof, row_idx=None, col_idx=None, KE_UNIT=KE_UNIT_3D, free=free.astype(np.int32),
                         F=F, ndof=ndof, backend="cupy", enable_warm_start=True, enable_matrix_free=True,
                         enable_fused_cuda=False, enable_matfree_gmg=True, matfree_gmg_levels=4,
                         gmg_fine_smoother=prec, gmg_smoother_type="chebyshev", grid_dims=nel, cg_tol=1e-8,
                         cg_maxiter=800, enable_profiling=True)
            rho = np.full(edof.shape[0], 0.3)
            comps, iters, rhos, dcs = [], [], [], []
            for _ in range(3):
                c, dc = s.solve(rho, penal=3.0)
                comps.append(c)
                iters.append(s.last_cg_iters)
                dcs.append(dc)
                rho = _oc_update(rho, dc, 0.3, 0.2, 1e-3)
                rhos.append(rho)
        d[f"compliance_{prec}"] = np.array(comps)
        d[f"iters_{prec}"] = np.array(iters)
        d[f"rho_{prec}"] = np.stack(rhos)
        d[f"dc_{prec}"] = np.stack(dcs)
    np.savez_compressed(HERE / "solverv4.npz", **d)

    # ---- OC on seeded inputs ----------------------------------------------
    d = {}
    rng = np.random.default_rng(3)
    for k, (n, vf, mv) in enumerate([(1728, 0.3, 0.2), (5000, 0.25, 0.1), (64, 0.5, 0.05)]):
        rho = rng.uniform(0.001, 1.0, n)
        dc = -rng.gamma(1.0, 1.0, n) * 10.0 ** rng.uniform(-6, 1, n)
        dc[::17] = 0.0  # exercises the min(dc, -1e-12) guard
        d[f"rho_{k}"] = rho
        d[f"dc_{k}"] = dc
        d[f"vf_{k}"] = np.array(vf)
        d[f"move_{k}"] = np.array(mv)
        d[f"out_{k}"] = _oc_update(rho, dc, vf, mv, 1e-3)
    np.savez_compressed(HERE / "oc.npz", **d)

    # ---- filters -----------------------------------------------------------
    d = {}
    for nel, rmin in [((24, 12, 6), 1.5), ((7, 5, 3), 2.0), ((6, 4, 3), 2.3)]:
        tag = "x".join(map(str, nel)) + f"_r{rmin}"
        d.update(_csr(f"H_{tag}", _build_density_filter(nel[0], nel[1], rmin, nel[2])))
    d["dense_432_r1.5"] = tg.DensityFilter((4, 3, 2), radius=1.5).matrix()
    d["dense_322_r1.5"] = tg.DensityFilter((3, 2, 2), radius=1.5).matrix()
    np.savez_compressed(HERE / "filter.npz", **d)

    # ---- run_simp, 24x12x6 cantilever --------------------------------------
    nel = (24, 12, 6)
    fixed, free, F, ndof = cantilever_bc(nel)
    params = SIMPParams(nelx=24, nely=12, nelz=6, volfrac=0.3, rmin=1.5, move=0.2, max_iter=3, min_iter=3,
                        use_heaviside=False)
    res = run_simp(params, verbose=False, bc_override=lambda a, b, c: (fixed, free, F))
    np.savez_compressed(HERE / "run_simp.npz", compliance=np.array(res["compliance_history"]),
                        final=np.array(res["final_compliance"]), rho_final=res["rho_final"])
    heaviside_fixtures(ref_root)
    checkpoint_fixtures(ref_root)
    wcycle_fixtures(ref_root)
    control_fixtures(ref_root)
    resume_fixtures(ref_root)
    print("golden fixtures written to", HERE)


def resume_fixtures(ref_root) -> None:
    import tempfile

    _setup(Path(ref_root))
    from gpu_fem.pub_simp_solver import SIMPParams, run_simp

    d = {}
    with tempfile.TemporaryDirectory() as tmp:
        for leg, max_iter in (("a", 4), ("b", 7)):
            params = SIMPParams(nelx=16, nely=8, nelz=4, volfrac=0.3, rmin=1.5, move=0.2, max_iter=max_iter,
                                min_iter=max_iter, use_heaviside=True, beta_init=2.0, checkpoint_dir=tmp,
                                checkpoint_every=2)
            with redirect_stdout(io.StringIO()):
                res = run_simp(params, verbose=False)
            d[f"compliance_{leg}"] = np.array(res["compliance_history"])
            d[f"rho_final_{leg}"] = res["rho_final"]
            d[f"n_iter_{leg}"] = np.array(res["n_iter"])
    np.savez_compressed(HERE / "run_simp_resume.npz", **d)


class ScriptedController:
    """Deterministic run_simp callback: the same script is replayed by the
    tests against the B200 driver."""

    def initial_action(self, params):
        return {"move": 0.15}

    def __call__(self, state, rho_new):
        if state.iteration == 2:
            return {"beta": 4.0, "penal": 3.5}
        if state.iteration == 4:
            return {"restart": True, "move": 0.1}
        if state.iteration == 6:
            return {"stop": True}
        return None

    def finalize_tail(self, params):
        return {"enabled": True, "tail_iters": 2, "penal": 4.0, "move": 0.05, "beta": 8.0, "rmin": 1.2}


def control_fixtures(ref_root) -> None:
    _setup(Path(ref_root))
    from gpu_fem.pub_simp_solver import SIMPParams, run_simp

    params = SIMPParams(nelx=16, nely=8, nelz=4, volfrac=0.3, rmin=1.5, move=0.2, max_iter=10, min_iter=3,
                        use_heaviside=True, beta_init=1.0, max_gray_for_best=0.9)
    with redirect_stdout(io.StringIO()):
        res = run_simp(params, callback=ScriptedController(), verbose=False)
    log = res["params_log"]
    d = {"compliance": np.array(res["compliance_history"]), "rho_final": res["rho_final"],
         "best_rho": res["best_rho"], "best_compliance": np.array(res["best_compliance"]),
         "best_iteration": np.array(res["best_iteration"]), "final_compliance": np.array(res["final_compliance"]),
         "best_is_valid": np.array(int(res["best_is_valid"])), "n_iter": np.array(res["n_iter"]),
         "log_iter": np.array([r["iter"] for r in log]), "log_tail": np.array([r["phase"] == "tail" for r in log]),
         "log_penal": np.array([r["penal"] for r in log]), "log_rmin": np.array([r["rmin"] for r in log]),
         "log_move": np.array([r["move"] for r in log]), "log_beta": np.array([r["beta"] for r in log]),
         "log_gray": np.array([r["grayness"] for r in log]), "log_vf": np.array([r["volume_fraction"] for r in log]),
         "pre_valid_best_compliance": np.array(res["pre_valid_best_compliance"])}
    np.savez_compressed(HERE / "run_simp_control.npz", **d)


def wcycle_fixtures(ref_root) -> None:
    _setup(Path(ref_root))
    import cupy as cp
    import gpu_fem.multigrid_v4 as mg
    import gpu_fem.solver_v2 as sv2
    from gpu_fem.pub_simp_solver import KE_UNIT_3D, _edof_table_3d

    d = {}
    for nel, nlev in [((24, 12, 6), 4), ((7, 5, 3), 3)]:
        tag = "x".join(map(str, nel))
        edof = _edof_table_3d(*nel)
        fixed, free, F, ndof = cantilever_bc(nel)
        rng = np.random.default_rng(11)
        rho = rng.uniform(0.05, 1.0, edof.shape[0])  # the galerkin.npz density
        E = 1e-9 + (1 - 1e-9) * rho**3
        free_gpu = cp.asarray(free.astype(np.int32))
        op = sv2.MatrixFreeKff(cp.asarray(edof), cp.asarray(KE_UNIT_3D), free_gpu, len(free), ndof)
        with redirect_stdout(io.StringIO()):
            g = mg.GalerkinMatFreeGMG(mf_op=op, free=free.astype(np.int32), free_gpu=free_gpu, nelx=nel[0],
                                      nely=nel[1], nelz=nel[2], KE_UNIT=KE_UNIT_3D, n_levels=nlev,
                                      fine_smoother="fp64", fine_smoother_degree=2, cycle_type="w")
            g.setup(cp.asarray(E))
        r = np.random.default_rng(12).standard_normal(len(free))
        d[f"rho_{tag}"] = rho
        d[f"r_{tag}"] = r
        d[f"z_{tag}"] = np.asarray(g.apply(cp.asarray(r)))
        Fd = cp.asarray(F[free])
        x, it, ok = sv2._cupy_pcg(lambda v: op.matvec(v, cp.asarray(E)), Fd, g.apply, tol=1e-8, maxiter=500)
        d[f"pcg_x_{tag}"] = np.asarray(x)
        d[f"pcg_it_{tag}"] = np.array(it)
    np.savez_compressed(HERE / "wcycle.npz", **d)


def checkpoint_fixtures(ref_root) -> None:
    import shutil
    import tempfile

    _setup(Path(ref_root))
    from gpu_fem.pub_simp_solver import SIMPParams, run_simp

    nel = (24, 12, 6)
    fixed, free, F, ndof = cantilever_bc(nel)
    with tempfile.TemporaryDirectory() as d:
        params = SIMPParams(nelx=24, nely=12, nelz=6, volfrac=0.3, rmin=1.5, move=0.2, max_iter=2, min_iter=2,
                            use_heaviside=False, checkpoint_dir=d, checkpoint_every=1)
        with redirect_stdout(io.StringIO()):
            run_simp(params, verbose=False, bc_override=lambda a, b, c: (fixed, free, F))
        for ext in (".npz", ".json"):
            shutil.copy(Path(d) / f"ckpt_24x12x6_cantilever{ext}", HERE / f"ckpt_24x12x6_cantilever{ext}")


def heaviside_fixtures(ref_root) -> None:
    _setup(Path(ref_root))
    from gpu_fem.pub_simp_solver import SIMPParams, run_simp

    nel = (24, 12, 6)
    fixed, free, F, ndof = cantilever_bc(nel)
    d = {}
    for beta in (1.0, 8.0):
        params = SIMPParams(nelx=24, nely=12, nelz=6, volfrac=0.3, rmin=1.5, move=0.2, max_iter=3, min_iter=3,
                            use_heaviside=True, beta_init=beta, eta=0.5)
        with redirect_stdout(io.StringIO()):
            res = run_simp(params, verbose=False, bc_override=lambda a, b, c: (fixed, free, F))
        tag = f"b{int(beta)}"
        d[f"compliance_{tag}"] = np.array(res["compliance_history"])
        d[f"rho_final_{tag}"] = res["rho_final"]
    np.savez_compressed(HERE / "run_simp_heaviside.npz", **d)


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("ref_root", nargs="?", default="/root/reference")
    ap.add_argument("--only", choices=["heaviside", "checkpoint", "wcycle", "control", "resume"], default=None)
    a = ap.parse_args()
    if a.only == "heaviside":
        heaviside_fixtures(a.ref_root)
    elif a.only == "checkpoint":
        checkpoint_fixtures(a.ref_root)
    elif a.only == "wcycle":
        wcycle_fixtures(a.ref_root)
    elif a.only == "control":
        control_fixtures(a.ref_root)
    elif a.only == "resume":
        resume_fixtures(a.ref_root)
    else:
        main(a.ref_root)
