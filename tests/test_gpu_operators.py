"""The operator-level drop-in classes (MatrixFreeOperator, GMGPreconditioner)
against the reference's own outputs: MatrixFreeKff.matvec and
extract_diagonal (src/gpu_fem/solver_v2.py:1183-1252, fixture matvec.npz)
and GalerkinMatFreeGMG.setup/apply with _cupy_pcg
(src/gpu_fem/multigrid_v4.py:657-844, solver_v2.py:552-624, fixture
galerkin.npz). Tolerances as in the context-level parity tests: FP64
round-off for the operator and the V-cycle, +-1 PCG iteration.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import fem

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("tag,nel", [("24x12x6", (24, 12, 6)), ("7x5x3", (7, 5, 3))])
def test_matrix_free_operator_matches_reference(cuda_dev, tag, nel):
    from topogpu_b200.operators import MatrixFreeOperator

    g = load_golden("matvec")
    bc = fem.cantilever_bc(nel)
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    op = MatrixFreeOperator(nel, mask, bc.F)
    E = torch.tensor(fem.simp_modulus(g[f"rho_{tag}"]), device=DEV)
    u = np.zeros(bc.ndof)
    u[bc.free] = g[f"u_{tag}"]
    y = op.matvec(torch.tensor(u, device=DEV), E).cpu().numpy()
    assert _rel(y[bc.free], g[f"y64_{tag}"]) < 1e-13
    assert np.all(y[bc.fixed] == 0.0)
    d = op.extract_diagonal(E).cpu().numpy()
    np.testing.assert_allclose(d[bc.free], g[f"diag_{tag}"], rtol=1e-14)
    # the FP32 operator through the same class
    y32 = op.matvec(torch.tensor(u, dtype=torch.float32, device=DEV), E.float()).cpu().numpy()
    assert _rel(y32[bc.free], g[f"y64_{tag}"]) < 2e-6


@pytest.mark.parametrize("tag,nel,nlev", [("24x12x6", (24, 12, 6), 4), ("7x5x3", (7, 5, 3), 3)])
def test_gmg_preconditioner_matches_reference(cuda_dev, tag, nel, nlev):
    from topogpu_b200.operators import GMGPreconditioner

    g = load_golden("galerkin")
    bc = fem.cantilever_bc(nel)
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    pre = GMGPreconditioner(nel, mask, bc.F, n_levels=nlev, precision="fp64", smoother="reference")
    E = torch.tensor(fem.simp_modulus(g[f"rho_{tag}"]), device=DEV)
    assert pre.setup(E) is pre
    info = pre.info
    np.testing.assert_allclose(info["lambda_max"][:-1], g[f"lam_{tag}"][:-1], rtol=1e-9)
    r = np.zeros(bc.ndof)
    r[bc.free] = g[f"r_{tag}"]
    z = pre.apply(torch.tensor(r, device=DEV)).cpu().numpy()
    assert _rel(z[bc.free], g[f"z_{tag}"]) < 1e-10
    assert np.all(z[bc.fixed] == 0.0)
    x, it, ok = pre.pcg(torch.tensor(bc.F, device=DEV), tol=1e-8, maxiter=500)
    assert ok and abs(it - int(g[f"pcg_it_{tag}"])) <= 1
    assert _rel(x.cpu().numpy()[bc.free], g[f"pcg_x_{tag}"]) < 1e-9
