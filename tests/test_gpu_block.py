"""Block PCG: several load cases on one density field (configuration 4a:
seeded unit point loads at random x = nelx face nodes in random unit
directions). The reference solves one load case per PCG, so each column is
checked against the per-case FP64 direct solve of the oracle (small mesh) and
against per-case single-RHS solves (96x48x48)."""

import dataclasses
import time

import numpy as np
import pytest
import torch

from oracle import fem
from topogpu_b200.bc import face_point_loads
from topogpu_b200.context import TopoContext
from topogpu_b200.state import StateSolver


def point_loads(nel, k, seed):
    return face_point_loads(nel, k, seed)


def _rho(n, seed):
    return np.random.default_rng(seed).uniform(0.05, 1.0, n)


@pytest.mark.gpu
def test_block_pcg_columns_match_direct_solves(cuda_dev):
    nel = (24, 12, 6)
    bc = fem.cantilever_bc(nel)
    rho = _rho(int(np.prod(nel)), 21)
    E = fem.simp_modulus(rho)
    B = point_loads(nel, 4, 22)
    ctx = TopoContext(nel, n_levels=3, mode="fp64")
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    ctx.set_problem(torch.tensor(mask, device="cuda"), torch.tensor(bc.F, device="cuda"))
    ctx.gmg_setup(torch.tensor(E, device="cuda"))
    Bt = torch.tensor(B, device="cuda")
    X = torch.zeros_like(Bt)
    it, rr, ok = ctx.block_pcg(Bt, X, tol=1e-10, maxiter=500)
    assert ok and max(rr) <= 1e-10, (it, rr)
    Xh = X.cpu().numpy()
    for j in range(4):
        ref = fem.direct_solve(E, nel, dataclasses.replace(bc, F=np.where(mask == 1, B[j], 0.0)))
        assert np.linalg.norm(Xh[j] - ref) <= 1e-8 * np.linalg.norm(ref), j
    # and against four single-RHS PCG solves on the same hierarchy
    single = 0
    for j in range(4):
        x = torch.zeros(bc.ndof, dtype=torch.float64, device="cuda")
        its, _, oks = ctx.pcg(Bt[j] * torch.tensor(mask, device="cuda"), x, tol=1e-10, maxiter=500)
        assert oks
        single += its
        assert float((x - X[j]).norm() / x.norm()) < 1e-8
    print(f"block PCG {it} iterations for 4 loads; single-RHS PCG {single} in total")
    ctx.close()


@pytest.mark.gpu
def test_block_pcg_config4a_mixed_vs_fp64(cuda_dev):
    nel = (96, 48, 48)
    bc = fem.cantilever_bc(nel)
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    rho = _rho(int(np.prod(nel)), 31)
    B = point_loads(nel, 8, 32)
    out = {}
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-5)):
        st = StateSolver(nel, mask, bc.F, n_levels=4, precision=prec, tol=tol, maxiter=800, fine_degree=3,
                         device="cuda")
        st.solve_block(rho, B)  # warm-up (workspaces, graphs)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        comp, U = st.solve_block(rho, B)
        torch.cuda.synchronize()
        out[prec] = (comp, st.last_cg_iters, time.perf_counter() - t0, st.last_converged)
        if prec == "mixed":
            # eight single-RHS solves on the same hierarchy for the timing comparison
            t0 = time.perf_counter()
            its = 0
            for j in range(8):
                x = torch.zeros(bc.ndof, dtype=torch.float64, device="cuda")
                i1, _, okj = st.ctx.pcg(torch.tensor(B[j] * mask, device="cuda"), x, tol, 800)
                assert okj
                its += i1
            torch.cuda.synchronize()
            out["single"] = (its, time.perf_counter() - t0)
        st.close()
    c64, cm = np.array(out["fp64"][0]), np.array(out["mixed"][0])
    assert out["fp64"][3] and out["mixed"][3]
    rel = np.abs(cm - c64) / np.abs(c64)
    print(f"8 load cases: block PCG fp64 {out['fp64'][1]} it / {out['fp64'][2] * 1e3:.1f} ms, "
          f"mixed {out['mixed'][1]} it / {out['mixed'][2] * 1e3:.1f} ms, "
          f"8 single mixed solves {out['single'][0]} it / {out['single'][1] * 1e3:.1f} ms; "
          f"max compliance rel err {rel.max():.2e}")
    assert rel.max() < 1e-4
