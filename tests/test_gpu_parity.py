"""GPU parity: libtopo_b200.so against the oracle and the reference fixtures.

Every test calls the CUDA path through the C ABI (via topogpu_b200.context)
on seeded inputs small enough for the oracle, and states its tolerance:
bit-exact for index work (filter neighbour sets, OC decisions), FP64
round-off for FP64 arithmetic, and the FP32 / BF16 bounds for reduced
precision.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import csr_from, load_golden
from oracle import design, fem, gmg, krylov, simp

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _ctx(nel, mode="fp64", n_levels=1, bc=None, smoother="reference", **kw):
    from topogpu_b200.context import TopoContext

    bc = bc or fem.cantilever_bc(nel)
    ctx = TopoContext(nel, n_levels=n_levels, mode=mode, smoother=smoother, **kw)
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    ctx.set_problem(torch.tensor(mask, device=DEV), torch.tensor(bc.F, device=DEV))
    return ctx, bc, mask


def _t(a, dtype=torch.float64):
    return torch.tensor(np.asarray(a), dtype=dtype, device=DEV)


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("tag,nel", [("24x12x6", (24, 12, 6)), ("7x5x3", (7, 5, 3))])
def test_matvec_fp64_fp32_bf16(cuda_dev, tag, nel):
    g = load_golden("matvec")
    ctx, bc, mask = _ctx(nel)
    E = fem.simp_modulus(g[f"rho_{tag}"])
    u = np.zeros(bc.ndof)
    u[bc.free] = g[f"u_{tag}"]
    y64 = ctx.matvec(_t(u), _t(E)).cpu().numpy()
    ref = g[f"y64_{tag}"]
    assert _rel(y64[bc.free], ref) < 1e-13
    assert np.all(y64[bc.fixed] == 0.0)
    y32 = ctx.matvec(_t(u, torch.float32), _t(E, torch.float32)).cpu().numpy()
    assert _rel(y32[bc.free], ref) < 2e-6
    # BF16 input (u stored in bf16), FP32 accumulation: compare with the
    # oracle's emulation of the same rounding, then with FP64.
    ub = torch.tensor(u, dtype=torch.float32, device=DEV).to(torch.bfloat16)
    yb = ctx.matvec(ub, _t(E, torch.float32)).cpu().numpy()
    emu = fem.matvec_full(fem.bf16_round(u), E.astype(np.float32), nel, "bf16")
    emu[bc.fixed] = 0.0
    assert _rel(yb, emu) < 1e-5
    assert _rel(yb[bc.free], ref) < 2e-2


def test_matvec_large_grid_against_assembled(cuda_dev):
    nel = (33, 17, 40)  # several blocks in every direction, ragged edges
    bc = fem.cantilever_bc(nel)
    ctx, _, _ = _ctx(nel, bc=bc)
    rng = np.random.default_rng(5)
    E = fem.simp_modulus(rng.uniform(0.001, 1.0, int(np.prod(nel))))
    u = np.zeros(bc.ndof)
    u[bc.free] = rng.standard_normal(len(bc.free))
    y = ctx.matvec(_t(u), _t(E)).cpu().numpy()
    ref = fem.matvec_full(u, E, nel)
    ref[bc.fixed] = 0.0
    assert _rel(y, ref) < 1e-13


@pytest.mark.parametrize("tag,nel", [("24x12x6", (24, 12, 6)), ("7x5x3", (7, 5, 3))])
def test_diagonal(cuda_dev, tag, nel):
    g = load_golden("matvec")
    ctx, bc, _ = _ctx(nel)
    E = fem.simp_modulus(g[f"rho_{tag}"])
    d = ctx.diag(_t(E)).cpu().numpy()
    np.testing.assert_allclose(d[bc.free], g[f"diag_{tag}"], rtol=1e-14)


def test_sensitivity_and_compliance(cuda_dev):
    nel = (11, 6, 5)
    ctx, bc, _ = _ctx(nel)
    rng = np.random.default_rng(9)
    rho = rng.uniform(0.05, 1.0, int(np.prod(nel)))
    u = rng.standard_normal(bc.ndof)
    u[bc.fixed] = 0.0
    dc = ctx.sensitivity(_t(u), _t(rho)).cpu().numpy()
    np.testing.assert_allclose(dc, fem.sensitivity(u, rho, nel), rtol=1e-12, atol=1e-14)
    dc32 = ctx.sensitivity(_t(u, torch.float32), _t(rho)).cpu().numpy()
    np.testing.assert_allclose(dc32, fem.sensitivity(u.astype(np.float32).astype(np.float64), rho, nel), rtol=1e-12,
                               atol=1e-14)
    assert abs(ctx.dot(_t(bc.F), _t(u)) - bc.F @ u) < 1e-12 * max(1.0, abs(bc.F @ u))


@pytest.mark.parametrize("nel,rmin", [((24, 12, 6), 1.5), ((7, 5, 3), 2.0), ((6, 4, 3), 2.3)])
def test_filter_and_transpose(cuda_dev, nel, rmin):
    g = load_golden("filter")
    H = csr_from(g, "H_" + "x".join(map(str, nel)) + f"_r{rmin}")
    ctx, _, _ = _ctx(nel)
    x = np.random.default_rng(1).uniform(0, 1, H.shape[0])
    y = ctx.filter(rmin, _t(x)).cpu().numpy()
    np.testing.assert_allclose(y, H @ x, rtol=1e-14, atol=1e-15)
    yt = ctx.filter(rmin, _t(x), transpose=True).cpu().numpy()
    np.testing.assert_allclose(yt, H.T @ x, rtol=1e-14, atol=1e-15)
    # uniform density is preserved (rows sum to one)
    np.testing.assert_allclose(ctx.filter(rmin, _t(np.ones(H.shape[0]))).cpu().numpy(), 1.0, atol=1e-14)


def test_oc_update_bit_exact(cuda_dev):
    g = load_golden("oc")
    for k in range(3):
        n = len(g[f"rho_{k}"])
        ctx, _, _ = _ctx((n, 1, 1))
        out, ev = ctx.oc(_t(g[f"rho_{k}"]), _t(g[f"dc_{k}"]), float(g[f"vf_{k}"]), float(g[f"move_{k}"]))
        assert np.array_equal(out.cpu().numpy(), g[f"out_{k}"]), k
        _, ev_ref = design.oc_update(g[f"rho_{k}"], g[f"dc_{k}"], float(g[f"vf_{k}"]), float(g[f"move_{k}"]))
        assert ev == ev_ref


def test_oc_filtered_matches_oracle(cuda_dev):
    nel = (24, 12, 6)
    H = design.filter_matrix(nel, 1.5)
    rng = np.random.default_rng(4)
    n = H.shape[0]
    rho = rng.uniform(0.01, 1.0, n)
    dc = -rng.gamma(1.0, 1.0, n)
    dv = H.T @ np.ones(n)
    ref, kref = design.oc_update_filtered(rho, dc, dv, 0.3, 0.2, H)
    ctx, _, _ = _ctx(nel)
    colsum = ctx.filter(1.5, _t(np.ones(n)), transpose=True)
    out, k = ctx.oc_filtered(_t(rho), _t(dc), _t(dv), colsum, 0.3, 0.2)
    assert k == kref
    assert np.array_equal(out.cpu().numpy(), ref)


@pytest.mark.parametrize("tag,nel,nlev", [("24x12x6", (24, 12, 6), 4), ("7x5x3", (7, 5, 3), 3)])
def test_vcycle_fp64_matches_reference(cuda_dev, tag, nel, nlev):
    """One V-cycle of the whole hierarchy (level-1 Galerkin, R.A.P, transfers,
    Chebyshev, spectral bounds, coarsest Cholesky) against the reference's."""
    g = load_golden("galerkin")
    ctx, bc, _ = _ctx(nel, n_levels=nlev)
    E = fem.simp_modulus(g[f"rho_{tag}"])
    ctx.gmg_setup(_t(E))
    info = ctx.gmg_info()
    np.testing.assert_allclose(info["lambda_max"][:-1], g[f"lam_{tag}"][:-1], rtol=1e-9)
    r = np.zeros(bc.ndof)
    r[bc.free] = g[f"r_{tag}"]
    z = ctx.gmg_apply(_t(r)).cpu().numpy()
    assert _rel(z[bc.free], g[f"z_{tag}"]) < 1e-10
    assert np.all(z[bc.fixed] == 0.0)
    for lv in range(1, nlev):
        assert info["n_free"][lv] == len(g[f"free{lv}_{tag}"])


@pytest.mark.parametrize("nel,nlev", [((24, 12, 6), 2), ((32, 16, 16), 2)])
def test_multi_panel_coarsest_factor_matches_oracle(cuda_dev, nel, nlev):
    """A coarsest system of many 32-column panels (1,008 and 3,888 free DoFs)
    factorised and inverted on the device: the
    V-cycle against the oracle's, whose coarsest solve is scipy's dense
    Cholesky (dense_chol_max raised to cover it)."""
    bc = fem.cantilever_bc(nel)
    rho = np.random.default_rng(9).uniform(0.05, 1.0, int(np.prod(nel)))
    E = fem.simp_modulus(rho)
    h = gmg.GMG(nel, bc.free, n_levels=nlev, fine_prec="fp64", fine_degree=2, dense_chol_max=20000).setup(E)
    assert h.chol is not None
    ctx, _, _ = _ctx(nel, n_levels=nlev, bc=bc)
    ctx.gmg_setup(_t(E))
    assert ctx.gmg_info()["n_free"][-1] == len(h.free[-1]) > 1000 - 8
    r = np.random.default_rng(10).standard_normal(len(bc.free))
    rf = np.zeros(bc.ndof)
    rf[bc.free] = r
    z = ctx.gmg_apply(_t(rf)).cpu().numpy()
    assert _rel(z[bc.free], h.apply(r)) < 1e-10


def _stencil_to_csr(S, dims):
    """(27,3,3,nnodes) stencil -> CSR over all DoFs of the level grid."""
    import scipy.sparse as sp

    nx, ny, nz = dims
    I, J, K = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    nn = len(I)
    rows, cols, vals = [], [], []
    for k in range(27):
        dx, dy, dz = k // 9 - 1, (k // 3) % 3 - 1, k % 3 - 1
        ok = (I + dx >= 0) & (I + dx <= nx) & (J + dy >= 0) & (J + dy <= ny) & (K + dz >= 0) & (K + dz <= nz)
        n = np.nonzero(ok)[0]
        m = ((I[n] + dx) * (ny + 1) + J[n] + dy) * (nz + 1) + K[n] + dz
        for c in range(3):
            for d in range(3):
                rows.append(3 * n + c)
                cols.append(3 * m + d)
                vals.append(S[k, c, d, n])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(3 * nn, 3 * nn))


@pytest.mark.parametrize("tag,nel,nlev", [("24x12x6", (24, 12, 6), 4), ("7x5x3", (7, 5, 3), 3)])
def test_level_operators_match_reference(cuda_dev, tag, nel, nlev):
    """Level-1 Galerkin and R.A.P operators, entry by entry, against the
    reference's CSR matrices (free x free)."""
    g = load_golden("galerkin")
    ctx, bc, _ = _ctx(nel, n_levels=nlev)
    ctx.gmg_setup(_t(fem.simp_modulus(g[f"rho_{tag}"])))
    dims = gmg.level_dims(nel, nlev)
    for lv in range(1, nlev):
        free = g[f"free{lv}_{tag}"]
        K = _stencil_to_csr(ctx.level_operator(lv).cpu().numpy(), dims[lv])
        Kf = K[free][:, free]
        R = csr_from(g, f"K{lv}_{tag}")
        assert abs(Kf - R).max() <= 1e-12 * abs(R).max(), lv
        # nothing outside the free set
        mask = np.zeros(K.shape[0], dtype=bool)
        mask[free] = True
        assert abs(K[~mask]).max() == 0.0 if (~mask).any() else True


@pytest.mark.parametrize("tag,nel,nlev", [("24x12x6", (24, 12, 6), 4), ("7x5x3", (7, 5, 3), 3)])
def test_pcg_and_fgmres_fp64_match_reference(cuda_dev, tag, nel, nlev):
    g = load_golden("galerkin")
    ctx, bc, _ = _ctx(nel, n_levels=nlev)
    E = fem.simp_modulus(g[f"rho_{tag}"])
    ctx.gmg_setup(_t(E))
    b = _t(bc.F)
    x = torch.zeros_like(b)
    it, rr, ok = ctx.pcg(b, x, tol=1e-8, maxiter=500)
    # On 7x5x3 the reference's relative residual after 45 iterations is
    # 1.077e-8, 8% above the tolerance: a 1e-16 relative perturbation of K.u
    # in the oracle already moves the stop between 45 and 46 (FGMRES stays at
    # its count), so PCG is held to +-1 iteration and the solution to 1e-9.
    assert ok and abs(it - int(g[f"pcg_it_{tag}"])) <= 1 and rr < 1e-8
    assert _rel(x.cpu().numpy()[bc.free], g[f"pcg_x_{tag}"]) < 1e-9
    x2 = torch.zeros_like(b)
    it2, rr2, ok2 = ctx.fgmres(b, x2, tol=1e-8, maxiter=500, restart=32)
    assert ok2 and it2 == int(g[f"fgmres_it_{tag}"])
    assert _rel(x2.cpu().numpy()[bc.free], g[f"fgmres_x_{tag}"]) < 1e-9


@pytest.mark.parametrize("tag,nel,nlev", [("24x12x6", (24, 12, 6), 4), ("7x5x3", (7, 5, 3), 3)])
def test_wcycle_fp64_matches_reference(cuda_dev, tag, nel, nlev):
    """W-cycle (two coarse corrections per level, multigrid_v4.py:1010-1042)
    against GalerkinMatFreeGMG(cycle_type="w"): one application to 1e-10, and
    PCG on it. PCG with this W-cycle is sensitive to rounding (1e-14 noise in
    F moves the reference count over 39-41 and 141-162), so the count is held
    to a 15% band and the solution to 1e-6."""
    g = load_golden("wcycle")
    ctx, bc, _ = _ctx(nel, n_levels=nlev)
    ctx.set_cycle("w")
    ctx.gmg_setup(_t(fem.simp_modulus(g[f"rho_{tag}"])))
    r = np.zeros(bc.ndof)
    r[bc.free] = g[f"r_{tag}"]
    z = ctx.gmg_apply(_t(r)).cpu().numpy()
    assert _rel(z[bc.free], g[f"z_{tag}"]) < 1e-10
    x = torch.zeros(bc.ndof, dtype=torch.float64, device=DEV)
    it, rr, ok = ctx.pcg(_t(bc.F), x, tol=1e-8, maxiter=500)
    ref_it = int(g[f"pcg_it_{tag}"])
    assert ok and rr < 1e-8 and abs(it - ref_it) <= max(2, 0.15 * ref_it)
    assert _rel(x.cpu().numpy()[bc.free], g[f"pcg_x_{tag}"]) < 1e-6
    ctx.set_cycle("v")  # back to the V-cycle: the galerkin.npz application again
    zv = ctx.gmg_apply(_t(r)).cpu().numpy()
    gv = load_golden("galerkin")
    rv = np.zeros(bc.ndof)
    rv[bc.free] = gv[f"r_{tag}"]
    assert _rel(ctx.gmg_apply(_t(rv)).cpu().numpy()[bc.free], gv[f"z_{tag}"]) < 1e-10
    assert not np.allclose(zv, z)


def test_wcycle_mixed_chebyshev_converges(cuda_dev):
    """The W-cycle with the default Chebyshev smoother and the mixed
    schedule solves to tolerance in no more iterations than the V-cycle."""
    from topogpu_b200.bc import cantilever_edge_load
    from topogpu_b200.state import StateSolver

    nel = (32, 16, 16)
    free, F = cantilever_edge_load(nel)
    rho = torch.as_tensor(np.random.default_rng(3).uniform(0.05, 1.0, int(np.prod(nel))), device=DEV)
    its = {}
    for cyc in ("v", "w"):
        st = StateSolver(nel, free, F, n_levels=3, precision="mixed", tol=1e-6, cycle_type=cyc)
        c, _ = st.solve(rho)
        assert st.last_converged
        its[cyc] = (st.last_cg_iters, float(c))
        st.close()
    assert its["w"][0] <= its["v"][0] + 2
    assert abs(its["w"][1] - its["v"][1]) < 1e-5 * abs(its["v"][1])


def test_pcg_warm_start_converged_up_front(cuda_dev):
    nel = (12, 6, 6)
    ctx, bc, _ = _ctx(nel, n_levels=3)
    E = fem.simp_modulus(np.full(int(np.prod(nel)), 0.4))
    ctx.gmg_setup(_t(E))
    x = torch.zeros(bc.ndof, dtype=torch.float64, device=DEV)
    ctx.pcg(_t(bc.F), x, tol=1e-10, maxiter=300)
    it, rr, ok = ctx.pcg(_t(bc.F), x, tol=1e-6, maxiter=300)
    assert ok and it == 0


def test_pcg_reports_cap(cuda_dev):
    nel = (12, 6, 6)
    ctx, bc, _ = _ctx(nel, n_levels=2)
    ctx.gmg_setup(_t(fem.simp_modulus(np.full(int(np.prod(nel)), 0.4))))
    x = torch.zeros(bc.ndof, dtype=torch.float64, device=DEV)
    it, rr, ok = ctx.pcg(_t(bc.F), x, tol=1e-14, maxiter=3)
    assert not ok and it == 3


def test_simp_solverv4_config0_fp64(cuda_dev):
    """Three SIMP iterations of the reference's SolverV4 path (no filter,
    move 0.2, tol 1e-8): compliance history within 1e-9 of the reference."""
    from topogpu_b200.state import StateSolver

    g = load_golden("solverv4")
    nel = (24, 12, 6)
    bc = fem.cantilever_bc(nel)
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    st = StateSolver(nel, mask, bc.F, n_levels=4, precision="fp64", tol=1e-8, maxiter=800, smoother="reference")
    rho = _t(np.full(1728, 0.3))
    comps = []
    for k in range(3):
        c, dc = st.solve(rho, 3.0)
        comps.append(c)
        rho, _ = st.ctx.oc(rho, dc, 0.3, 0.2, 1e-3)
        assert np.max(np.abs(rho.cpu().numpy() - g["rho_fp64"][k])) < 1e-7
    np.testing.assert_allclose(comps, g["compliance_fp64"], rtol=1e-9)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-5), ("fp32", 1e-4), ("mixed", 1e-4)])
def test_reduced_precision_compliance_vs_fp64_oracle(cuda_dev, precision, tol):
    """Compliance of each precision mode against the direct FP64 solve on a
    high-contrast random density (48x24x24, rho ~ U[0.05, 1] filtered with
    rmin 1.5): within 1e-4 relative at rtol 1e-5, the required bar. The Chebyshev smoother keeps every mode within
    a few tens of PCG iterations (the reference recurrence needs 93-140 in
    FP64 on this input and does not converge in FP32)."""
    from topogpu_b200.state import StateSolver

    nel = (48, 24, 24)
    bc = fem.cantilever_bc(nel)
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    rho = np.random.default_rng(2).uniform(0.05, 1.0, int(np.prod(nel)))
    rho = design.filter_matrix(nel, 1.5) @ rho
    u_ref = fem.direct_solve(fem.simp_modulus(rho), nel, bc)
    c_ref = bc.F @ u_ref
    st = StateSolver(nel, mask, bc.F, n_levels=4, precision=precision, fine_degree=3, tol=1e-5, maxiter=800)
    c, dc = st.solve(_t(rho), 3.0)
    assert st.last_converged and st.last_relres <= 1e-5
    assert st.last_cg_iters <= 40, st.last_cg_iters
    assert abs(c - c_ref) / abs(c_ref) < tol
    u = st.displacement().cpu().numpy()
    assert _rel(u, u_ref) < 1e-4
    dc_ref = fem.sensitivity(u_ref, rho, nel)
    assert _rel(dc.cpu().numpy(), dc_ref) < 1e-3


def test_mixed_solution_at_size_checked_by_oracle_operator(cuda_dev):
    """The 1M-element SIMP mesh (160x80x80 cantilever, filtered random
    density): the mixed-mode displacement (rtol 1e-5) and the FP64-mode one
    (rtol 1e-8) are checked with the oracle's own matrix-free FP64 K.u, so the
    bar does not rest on this library's FP64 path: true relative residual
    <= 5e-5 (mixed) and <= 1e-7 (FP64) on the free DoFs, and the mixed
    compliance within 1e-4 of the FP64 one (the required bar). A converged
    oracle solve at this size takes minutes on the host, so the oracle
    checks the residual instead."""
    from topogpu_b200.state import StateSolver

    nel = (160, 80, 80)
    bc = fem.cantilever_bc(nel)
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    rho0 = _t(np.random.default_rng(5).uniform(0.05, 1.0, int(np.prod(nel))))
    out = {}
    for precision, tol in (("mixed", 1e-5), ("fp64", 1e-8)):
        st = StateSolver(nel, mask, bc.F, n_levels=4, precision=precision, fine_degree=3, tol=tol, maxiter=800)
        rho = st.ctx.filter(1.5, rho0)
        c, _ = st.solve(rho, 3.0)
        assert st.last_converged and st.last_relres <= tol
        u = st.displacement().cpu().numpy()
        r = bc.F - fem.matvec_full(u, fem.simp_modulus(rho.cpu().numpy()), nel)
        out[precision] = (c, np.linalg.norm(r[bc.free]) / np.linalg.norm(bc.F[bc.free]))
        del st
        torch.cuda.empty_cache()
    print({k: (f"{v[0]:.10g}", f"{v[1]:.2e}") for k, v in out.items()})
    assert out["mixed"][1] <= 5e-5
    assert out["fp64"][1] <= 1e-7
    assert abs(out["mixed"][0] - out["fp64"][0]) / abs(out["fp64"][0]) < 1e-4


def test_run_simp_config0_filtered_fp64(cuda_dev):
    """Config 0 as specified (filter rmin 1.5, move 0.2, 3 OC iterations):
    compliance history of the reference's run_simp."""
    import topogpu_b200 as tg

    g = load_golden("run_simp")
    p = tg.gallery.benchmark_cantilever((24, 12, 6), volfrac=0.3, filter_radius=1.5)
    res = tg.SIMPSolver(backend="cuda", tol=1e-10, max_krylov=800, max_iter=3, move=0.2, precision="fp64",
                        use_filter=True).solve(p)
    comp = [r["compliance"] for r in res.history]
    np.testing.assert_allclose(comp, g["compliance"], rtol=1e-8)


def test_simpsolver_evidence_bundle(cuda_dev, tmp_path):
    import topogpu_b200 as tg

    p = tg.gallery.cantilever_3d(nel=(8, 4, 4), volfrac=0.30)
    res = tg.SIMPSolver(backend="cuda", max_iter=2, max_krylov=200).solve(p)
    b = res.save(tmp_path / "run")
    for f in ["summary.json", "history.csv", "rho_final.npy", "render_metadata.json", "ARTIFACT_MANIFEST.csv"]:
        assert (tmp_path / "run" / f).exists()
    h = res.history[-1]
    assert set(h) == {"iteration", "compliance", "outer_iters", "rho_mean", "rho_min", "rho_max", "grayness",
                      "wall_s", "outer_solver"}
    assert abs(h["rho_mean"] - 0.3) < 1e-6
    assert len(b.rows) == 4


@pytest.mark.gpu
def test_lagged_coarse_factor_same_solutions(cuda_dev):
    """With the one-setup-lagged coarsest factor (built in the background) the
    solves converge to the same compliances as with the synchronous factor."""
    from topogpu_b200.bc import cantilever_edge_load
    from topogpu_b200.state import StateSolver

    nel = (48, 24, 24)
    mask, F = cantilever_edge_load(nel)
    rng = np.random.default_rng(17)
    rhos = [torch.tensor(rng.uniform(0.05, 1.0, 48 * 24 * 24), device=DEV) for _ in range(4)]
    out = {}
    for lag in (False, True):
        st = StateSolver(nel, mask, F, n_levels=4, precision="mixed", tol=1e-6, device=DEV)
        st.ctx.set_coarse_lag(lag)
        comps = []
        for r in rhos:
            c, _ = st.solve(r)
            assert st.last_converged
            comps.append(c)
        out[lag] = np.array(comps)
        st.close()
    assert np.max(np.abs(out[True] - out[False]) / np.abs(out[False])) < 1e-5


@pytest.mark.gpu
def test_probe_quality_and_kappa_eff_match_oracle(cuda_dev):
    """probe_quality and the Lanczos kappa_eff of M K (multigrid_v4.py:606-655,
    821-832) on the reference V-cycle, against the same Lanczos run on the
    oracle hierarchy with the same start vector."""
    from topogpu_b200.state import StateSolver

    g = load_golden("galerkin")
    tag, nel, nlev = "24x12x6", (24, 12, 6), 4
    bc = fem.cantilever_bc(nel)
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    st = StateSolver(nel, mask, bc.F, n_levels=nlev, precision="fp64", smoother="reference", probe=True,
                     tol=1e-8, device=DEV)
    rho = g[f"rho_{tag}"]
    st.solve(rho)
    q = st.last_multigrid_quality
    assert q["finite"] and q["pd"] and q["z_norm"] > 0 and q["jacobi_norm"] > 0
    kappa = st.estimate_kappa_eff(30)
    # oracle: same start vector (torch generator, seed 0), compact free vectors
    h = gmg.GMG(nel, bc.free, n_levels=nlev, fine_prec="fp64", fine_degree=2).setup(fem.simp_modulus(rho))
    v = (torch.randn(bc.ndof, generator=torch.Generator().manual_seed(0), dtype=torch.float64).numpy())[bc.free]
    v /= np.linalg.norm(v)
    vp = np.zeros_like(v)
    al, be = [], []
    for j in range(30):
        w = h.apply(h.fine_op64(v))
        a = float(v @ w)
        al.append(a)
        w = w - a * v - (be[-1] * vp if j > 0 else 0.0)
        if j < 29:
            b = float(np.linalg.norm(w))
            be.append(b)
            vp, v = v, w / b
    eig = np.linalg.eigvalsh(np.diag(al) + np.diag(be, 1) + np.diag(be, -1))
    ref = eig[-1] / eig[eig > 0][0]
    assert abs(kappa - ref) <= 1e-6 * ref, (kappa, ref)
    st.close()


def test_different_element_stiffness_refused_while_shared_one_is_live(cuda_dev):
    """KE sits in constant memory shared by every context of a device: a
    context with another KE is refused while one with the default is alive,
    and a second context with the same KE is accepted."""
    from topogpu_b200.context import TopoContext
    from topogpu_b200.fem import KE_UNIT

    a = TopoContext((4, 2, 2), n_levels=1, mode="fp64")
    with pytest.raises(RuntimeError, match="different element stiffness"):
        TopoContext((4, 2, 2), n_levels=1, mode="fp64", KE=KE_UNIT * 2.0)
    b = TopoContext((4, 2, 2), n_levels=1, mode="fp64", KE=KE_UNIT.copy())
    # the reference's KE_UNIT_3D differs from this one in the last bits: same stiffness
    c = TopoContext((4, 2, 2), n_levels=1, mode="fp64", KE=load_golden("ke_edof")["KE"])
    assert a.ndof == b.ndof == c.ndof


def test_solverv4_class_matches_reference_fixture(cuda_dev):
    """tg.SolverV4 built with the reference's own constructor arguments
    (solver_v4.py:38-145, as in the solverv4.npz generator, with the
    reference's KE_UNIT_3D) and driven by the host OC: the reference's
    compliances to 1e-9 and densities to 1e-7."""
    import topogpu_b200 as tg

    g = load_golden("solverv4")
    ke = load_golden("ke_edof")["KE"]
    nel = (24, 12, 6)
    bc = fem.cantilever_bc(nel)
    s = tg.SolverV4(edof=None, row_idx=None, col_idx=None, KE_UNIT=ke, free=bc.free.astype(np.int32), F=bc.F,
                    ndof=bc.ndof, backend="cupy", enable_warm_start=True, enable_matrix_free=True,
                    enable_fused_cuda=False, enable_matfree_gmg=True, matfree_gmg_levels=4,
                    gmg_fine_smoother="fp64", gmg_smoother_type="chebyshev", grid_dims=nel, cg_tol=1e-8,
                    cg_maxiter=800, enable_profiling=True)
    rho = np.full(1728, 0.3)
    comps = []
    for k in range(3):
        c, dc = s.solve(rho, penal=3.0)
        comps.append(c)
        # PCG on this 131-iteration case is not reproducible to the iteration
        # (the reference V-cycle is only nearly symmetric): within 5%
        assert isinstance(dc, np.ndarray) and abs(s.last_cg_iters - int(g["iters_fp64"][k])) <= 0.05 * int(
            g["iters_fp64"][k]) + 1
        rho, _ = design.oc_update(rho, dc, 0.3, 0.2)
        assert np.max(np.abs(rho - g["rho_fp64"][k])) < 1e-7
    np.testing.assert_allclose(comps, g["compliance_fp64"], rtol=1e-9)
    assert s.last_outer_solver == "pcg" and s.last_timing
    s.close()
