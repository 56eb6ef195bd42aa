"""Pins the CPU oracle against fixtures produced by the unmodified reference.

The fixtures come from ``tests/golden/make_golden.py`` (reference code run on
a NumPy-backed CuPy stand-in). If the oracle agrees with them here, the GPU
parity tests that compare against the oracle inherit the reference's answers.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import csr_from, load_golden
from oracle import design, fem, gmg, krylov, simp


def test_ke_and_edof_bit_exact():
    g = load_golden("ke_edof")
    np.testing.assert_allclose(fem.KE_UNIT, g["KE"], rtol=0, atol=1e-15)
    assert np.array_equal(fem.edof_table((4, 3, 2)), g["edof_432"])
    assert np.array_equal(fem.edof_table((7, 5, 3)), g["edof_753"])


@pytest.mark.parametrize("tag,nel", [("24x12x6", (24, 12, 6)), ("7x5x3", (7, 5, 3))])
def test_matvec_and_diag(tag, nel):
    g = load_golden("matvec")
    bc = fem.cantilever_bc(nel)
    E = fem.simp_modulus(g[f"rho_{tag}"])
    y = fem.matvec_free(g[f"u_{tag}"], E, nel, bc.free, "fp64")
    ref = g[f"y64_{tag}"]
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-14
    y32 = fem.matvec_free(g[f"u_{tag}"].astype(np.float32), E.astype(np.float32), nel, bc.free, "fp32")
    assert np.linalg.norm(y32 - g[f"y32_{tag}"]) / np.linalg.norm(ref) < 1e-6
    d = fem.diagonal_full(E, nel)[bc.free]
    np.testing.assert_allclose(d, g[f"diag_{tag}"], rtol=1e-14)


def test_transfers_bit_exact():
    g = load_golden("transfer")
    pairs = [((24, 12, 6), (12, 6, 3)), ((12, 6, 3), (6, 3, 1)), ((6, 3, 1), (3, 1, 1)),
             ((7, 5, 3), (3, 2, 1)), ((3, 2, 1), (1, 1, 1)), ((1, 1, 1), (1, 1, 1))]
    for fine, coarse in pairs:
        tag = "x".join(map(str, fine)) + "_" + "x".join(map(str, coarse))
        P = gmg.scalar_prolongation(fine, coarse)
        P.sort_indices()
        R = csr_from(g, f"P_{tag}")
        assert np.array_equal(P.indptr, R.indptr) and np.array_equal(P.indices, R.indices)
        assert np.array_equal(P.data, R.data)  # powers of two: bit-exact
        bc = fem.cantilever_bc(fine)
        assert np.array_equal(gmg.injection_free(fine, coarse, bc.free), g[f"inj_{tag}"])


@pytest.mark.parametrize("tag,nel,nlev", [("24x12x6", (24, 12, 6), 4), ("7x5x3", (7, 5, 3), 3)])
def test_galerkin_hierarchy_and_vcycle(tag, nel, nlev):
    g = load_golden("galerkin")
    bc = fem.cantilever_bc(nel)
    E = fem.simp_modulus(g[f"rho_{tag}"])
    h = gmg.GMG(nel, bc.free, n_levels=nlev, fine_prec="fp64", fine_degree=2).setup(E)
    for lv in range(1, nlev):
        assert np.array_equal(h.free[lv], g[f"free{lv}_{tag}"])
        K = csr_from(g, f"K{lv}_{tag}")
        diff = abs(h.K[lv] - K).max()
        assert diff <= 1e-12 * abs(K).max(), (lv, diff)
    np.testing.assert_allclose(h.lam, g[f"lam_{tag}"], rtol=1e-10)
    z = h.apply(g[f"r_{tag}"])
    ref = g[f"z_{tag}"]
    assert np.linalg.norm(z - ref) / np.linalg.norm(ref) < 1e-10
    # Krylov on the same hierarchy
    A = h.fine_op64
    F = bc.F[bc.free]
    x, it, ok = krylov.pcg(A, F, h.apply, tol=1e-8, maxiter=500)
    assert ok and it == int(g[f"pcg_it_{tag}"])
    xr = g[f"pcg_x_{tag}"]
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-9
    x2, it2, ok2 = krylov.fgmres(A, F, h.apply, tol=1e-8, maxiter=500, restart=32)
    assert ok2 and it2 == int(g[f"fgmres_it_{tag}"])
    assert np.linalg.norm(x2 - g[f"fgmres_x_{tag}"]) / np.linalg.norm(xr) < 1e-9


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_solverv4_simp_config0(prec):
    g = load_golden("solverv4")
    nel = (24, 12, 6)
    bc = fem.cantilever_bc(nel)
    rho, comp, rhos = simp.simp_solverv4(nel, bc, 0.3, 3, move=0.2, fine_prec=prec, tol=1e-8, maxiter=800)
    if prec == "fp64":
        np.testing.assert_allclose(comp, g[f"compliance_{prec}"], rtol=1e-9)
        # design updates reproduce the reference's to FP64 round-off of the solve
        assert np.max(np.abs(np.stack(rhos) - g[f"rho_{prec}"])) < 1e-7
    else:
        # Step 1 converges (38 iterations in both); in steps 2-3 the reference
        # itself stalls at max_krylov=800 with the FP32 smoother at tol 1e-8,
        # so those iterates depend on rounding: hold them to the FP32 bar.
        np.testing.assert_allclose(comp[0], g["compliance_fp32"][0], rtol=1e-9)
        np.testing.assert_allclose(comp, g["compliance_fp32"], rtol=1e-4)


def test_oc_update_bit_exact():
    g = load_golden("oc")
    for k in range(3):
        out, _ = design.oc_update(g[f"rho_{k}"], g[f"dc_{k}"], float(g[f"vf_{k}"]), float(g[f"move_{k}"]))
        assert np.array_equal(out, g[f"out_{k}"])


def test_filter_index_sets_bit_exact_and_values():
    g = load_golden("filter")
    for nel, rmin in [((24, 12, 6), 1.5), ((7, 5, 3), 2.0), ((6, 4, 3), 2.3)]:
        tag = "x".join(map(str, nel)) + f"_r{rmin}"
        H = design.filter_matrix(nel, rmin)
        H.sort_indices()
        R = csr_from(g, f"H_{tag}")
        assert np.array_equal(H.indptr, R.indptr) and np.array_equal(H.indices, R.indices)
        np.testing.assert_allclose(H.data, R.data, rtol=1e-15, atol=0)
    np.testing.assert_allclose(design.dense_filter_matrix((4, 3, 2), 1.5), g["dense_432_r1.5"], rtol=1e-15)
    np.testing.assert_allclose(design.dense_filter_matrix((3, 2, 2), 1.5), g["dense_322_r1.5"], rtol=1e-15)


def test_run_simp_config0_known_answer():
    g = load_golden("run_simp")
    nel = (24, 12, 6)
    bc = fem.cantilever_bc(nel)
    rho, hist, cf, rpf = simp.simp_filtered(nel, bc, 0.3, 1.5, 3, move=0.2)
    np.testing.assert_allclose(hist, g["compliance"], rtol=1e-10)
    np.testing.assert_allclose(cf, float(g["final"]), rtol=1e-10)
    np.testing.assert_allclose(rpf, g["rho_final"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("tag,nel,nlev", [("24x12x6", (24, 12, 6), 4), ("7x5x3", (7, 5, 3), 3)])
def test_wcycle_against_reference(tag, nel, nlev):
    """GalerkinMatFreeGMG(cycle_type="w") on the galerkin.npz hierarchies
    (multigrid_v4.py:1010-1042): one application and PCG to 1e-8."""
    g = load_golden("wcycle")
    bc = fem.cantilever_bc(nel)
    h = gmg.GMG(nel, bc.free, n_levels=nlev, fine_prec="fp64", fine_degree=2, cycle="w").setup(
        fem.simp_modulus(g[f"rho_{tag}"]))
    z = h.apply(g[f"r_{tag}"])
    assert np.linalg.norm(z - g[f"z_{tag}"]) / np.linalg.norm(g[f"z_{tag}"]) < 1e-10
    # PCG with this W-cycle is sensitive to rounding: 1e-14 relative noise in
    # F moves the count over 39-41 (24x12x6) and 141-162 (7x5x3), so the count
    # is held to a 15% band and the solution to the tolerance
    x, it, ok = krylov.pcg(h.fine_op64, bc.F[bc.free], h.apply, tol=1e-8, maxiter=500)
    ref_it = int(g[f"pcg_it_{tag}"])
    assert ok and abs(it - ref_it) <= max(2, 0.15 * ref_it)
    xr = g[f"pcg_x_{tag}"]
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-6


def test_run_simp_heaviside_known_answer():
    """The projected loop against run_simp with use_heaviside at beta 1 and 8
    (fixture made by tests/golden/make_golden.py --only heaviside)."""
    g = load_golden("run_simp_heaviside")
    nel = (24, 12, 6)
    bc = fem.cantilever_bc(nel)
    for beta in (1, 8):
        rho, hist, cf, rpf = simp.simp_projected(nel, bc, 0.3, 1.5, 3, float(beta), move=0.2)
        np.testing.assert_allclose(hist, g[f"compliance_b{beta}"], rtol=1e-10)
        # the bisection stops at a lambda bracket of 1e-9, so the last candidate
        # carries that much slack; the steep projection (slope up to beta/2)
        # amplifies it in the physical density
        np.testing.assert_allclose(rpf, g[f"rho_final_b{beta}"], rtol=1e-9, atol=1e-9)


def test_known_answer_uniform_density_compliance():
    """Known answer for the 24x12x6 cantilever at uniform density 0.3: the
    compliance F.u of the direct FP64 solve."""
    nel = (24, 12, 6)
    bc = fem.cantilever_bc(nel)
    u = fem.direct_solve(fem.simp_modulus(np.full(1728, 0.3)), nel, bc)
    assert abs(bc.F @ u - 399.9508808170127) < 1e-9


def test_heaviside_restatement_matches_reference_formulas():
    """The projection and its derivative against a central difference, and
    the beta -> 0 identity (pub_simp_solver.py:245-253)."""
    x = np.linspace(0.0, 1.0, 101)
    for beta in (1.0, 8.0, 32.0):
        h = design.heaviside(x, beta, 0.5)
        assert abs(h[0]) < 1e-15 and abs(h[-1] - 1.0) < 1e-15
        eps = 1e-6
        fd = (design.heaviside(x + eps, beta, 0.5) - design.heaviside(x - eps, beta, 0.5)) / (2 * eps)
        np.testing.assert_allclose(design.heaviside_deriv(x, beta, 0.5), fd, rtol=1e-6, atol=1e-8)
    assert np.array_equal(design.heaviside(x, 0.0, 0.5), x)
