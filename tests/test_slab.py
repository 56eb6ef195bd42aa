"""x-slab decomposition (topogpu_b200.slab) with 2 and 3 gloo ranks on CPU.

The per-rank arithmetic comes from the oracle (the slab's K u, and its
Schwarz piece as an exact sparse solve or an oracle V-cycle), so these tests
check the decomposition itself against the undivided oracle problem:
interface sums, owned-plane dot products, the symmetry of the assembled
preconditioner, and PCG converging to the global solution. Tolerances:
round-off (1e-12) for the matvec, dots and symmetry; the PCG tolerance for
the solution.
"""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleSlabOps:
    """SlabLocalOps from the oracle on one rank's slab."""

    def __init__(self, slab, bc, E, precond="exact"):
        import scipy.sparse.linalg as spla

        from oracle import fem, gmg

        self.fem, self.slab = fem, slab
        a, b = slab.element_range(slab.e0, slab.e1)
        self.E_op = E[a:b]
        self.mask = slab.local_free_mask(bc.free_mask())
        a, b = slab.element_range(slab.x_lo, slab.x_hi)
        E_ext = E[a:b]
        m_ext = slab.ext_free_mask(bc.free_mask())
        self.free_ext = np.flatnonzero(m_ext)
        self.n_ext = len(m_ext)
        self.off = slab.ext_offset()
        if precond == "exact":
            K = fem.assemble_K(E_ext, slab.ext_nel).tocsc()[self.free_ext][:, self.free_ext]
            self._solve = spla.splu(K.tocsc()).solve
        else:
            h = gmg.GMG(slab.ext_nel, self.free_ext, n_levels=2, fine_prec="fp64", fine_degree=2,
                        dense_chol_max=20000).setup(E_ext)
            self._solve = h.apply

    def matvec(self, u):
        import torch

        y = self.fem.matvec_full(u.numpy(), self.E_op, self.slab.local_nel) * self.mask
        return torch.as_tensor(y)

    def precondition(self, r):
        import torch

        n = self.slab.piece_ndof
        ext = np.zeros(self.n_ext)
        ext[self.off:self.off + n] = r.numpy()
        z = np.zeros(self.n_ext)
        z[self.free_ext] = self._solve(ext[self.free_ext])
        return torch.as_tensor(z[self.off:self.off + n].copy())


def _bc_free_mask(bc):
    m = np.zeros(bc.ndof, dtype=np.uint8)
    m[bc.free] = 1
    return m


def _rank(rank, world, port, nel, precond, out, coarse_levels=0, overlap=0, balanced=False):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import fem
        from topogpu_b200.slab import Slab, SlabPCG, all_dots

        bc = fem.cantilever_bc(nel)
        bc.free_mask = lambda: _bc_free_mask(bc)
        rho = np.random.default_rng(5).uniform(0.1, 1.0, int(np.prod(nel)))
        E = fem.simp_modulus(rho)
        slab = Slab.of(nel, rank, world, overlap)
        ops = OracleSlabOps(slab, bc, E, precond)
        coarse, res_a0 = None, None
        if coarse_levels:
            from topogpu_b200.slab import SlabCoarse, coarse_prolongation

            P0 = coarse_prolongation(nel, _bc_free_mask(bc), coarse_levels)
            a0, b0 = slab.dof_range()
            P = torch.as_tensor(P0[a0:b0].toarray())
            A0 = SlabCoarse.galerkin(slab, P, ops.matvec, dist)
            coarse = SlabCoarse(slab, P, A0, dist)
            # the summed Galerkin operator is the global P0^T K P0
            K = fem.assemble_K(E, nel)
            A0_ref = (P0.T @ K @ P0).toarray()
            res_a0 = float(np.abs(A0.numpy() - A0_ref).max() / np.abs(A0_ref).max())
        pcg = SlabPCG(slab, ops, dist, coarse=coarse, balanced=balanced)
        a, b = slab.dof_range()
        mask = _bc_free_mask(bc)
        rng = np.random.default_rng(1)
        u = rng.standard_normal(bc.ndof) * mask
        v = rng.standard_normal(bc.ndof) * mask
        res = {}
        # 1. distributed K u against the global operator on this rank's planes
        y = pcg.apply_K(torch.as_tensor(u[a:b].copy())).numpy()
        yg = fem.matvec_full(u, E, nel) * mask
        res["matvec"] = np.abs(y - yg[a:b]).max() / np.abs(yg).max()
        # 2. owned-plane dots
        (d,) = all_dots([(torch.as_tensor(u[a:b].copy()), torch.as_tensor(v[a:b].copy()))], pcg.w, dist, world)
        res["dot"] = abs(d - u @ v) / abs(u @ v)
        # 3. the assembled preconditioner is symmetric
        mu = pcg.apply_M(torch.as_tensor(u[a:b].copy()))
        mv = pcg.apply_M(torch.as_tensor(v[a:b].copy()))
        vmu, umv = all_dots([(torch.as_tensor(v[a:b].copy()), mu), (torch.as_tensor(u[a:b].copy()), mv)], pcg.w,
                            dist, world)
        res["sym"] = abs(vmu - umv) / abs(vmu)
        (umu,) = all_dots([(torch.as_tensor(u[a:b].copy()), mu)], pcg.w, dist, world)
        res["pos"] = umu
        # 4. PCG to the global direct solution
        F = torch.as_tensor((bc.F * mask)[a:b].copy())
        x, it, rr, ok = pcg.solve(F, tol=1e-10, maxiter=400)
        U = fem.direct_solve(E, nel, bc)
        res["x_err"] = np.abs(x.numpy() - U[a:b]).max() / np.abs(U).max()
        (c,) = all_dots([(F, x)], pcg.w, dist, world)
        res["compliance_err"] = abs(c - bc.F @ U) / abs(bc.F @ U)
        res["iters"], res["ok"] = it, ok
        res["a0"] = res_a0
        out[rank] = res
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run(world, nel, precond, coarse_levels=0, overlap=0, balanced=False):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, nel, precond, out, coarse_levels, overlap, balanced), nprocs=world,
                 join=True)
        return dict(out)


def test_partition_and_slab_geometry():
    from topogpu_b200.slab import Slab, partition

    assert partition(10, 3) == [(0, 4), (4, 7), (7, 10)]
    with pytest.raises(ValueError):
        partition(2, 3)
    s = Slab.of((12, 4, 4), 1, 3)
    assert (s.e0, s.e1, s.x_lo, s.x_hi) == (4, 8, 3, 9)
    assert s.n_planes == 5 and s.plane_dofs == 75 and s.ndof == 375
    assert s.ext_nel == (6, 4, 4) and s.ext_offset() == 75
    w = s.owned_mask()
    assert float(w[:75].sum()) == 0 and float(w[75:].sum()) == 300
    m = s.ext_free_mask(np.ones(3 * 13 * 25, dtype=np.uint8))
    assert m[:75].sum() == 0 and m[-75:].sum() == 0 and m[75:-75].all()


@pytest.mark.parametrize("world,precond", [(1, "exact"), (2, "exact"), (3, "exact"), (3, "gmg")])
def test_slab_pcg_matches_undivided_problem(world, precond):
    nel = (12, 4, 4)
    res = _run(world, nel, precond)
    assert sorted(res) == list(range(world))
    iters = {r["iters"] for r in res.values()}
    assert len(iters) == 1  # every rank took the same steps
    for r in res.values():
        assert r["matvec"] < 1e-12 and r["dot"] < 1e-12 and r["sym"] < 1e-10 and r["pos"] > 0
        assert r["ok"] and r["x_err"] < 1e-7 and r["compliance_err"] < 1e-8
    # one rank with an exact piece is a direct solve; with more slabs the
    # one-level Schwarz preconditioner (no coarse space) needs more steps:
    # 30 / 42 / 46 iterations to 1e-10 for 2 / 3 / 4 slabs of this mesh
    # (66 / 76 with oracle V-cycles as the pieces)
    it = iters.pop()
    if precond == "exact":
        assert it == 1 if world == 1 else it <= 50
    else:
        assert it <= 90


def _iters(world, nel, precond, **kw):
    res = _run(world, nel, precond, **kw)
    for r in res.values():
        if kw.get("coarse_levels"):
            assert r["a0"] < 1e-12
        assert r["matvec"] < 1e-12 and r["sym"] < 1e-10 and r["pos"] > 0
        assert r["ok"] and r["x_err"] < 1e-7 and r["compliance_err"] < 1e-8
    its = {r["iters"] for r in res.values()}
    assert len(its) == 1  # every rank took the same steps
    return its.pop()


@pytest.mark.parametrize("precond", ["exact", "gmg"])
def test_two_level_balanced_schwarz_flattens_the_iteration_count(precond):
    """One overlap plane and the replicated coarse space (one factor-2
    coarsening of the whole mesh, its Galerkin operator summed from every
    rank's elements and checked against P0^T K P0) in the balanced form:
    going from 2 to 4 slabs costs at most 20% more PCG iterations, and at 4
    slabs it needs clearly fewer than the one-level form."""
    nel = (16, 4, 4)
    two = {w: _iters(w, nel, precond, coarse_levels=1, overlap=1, balanced=True) for w in (2, 4)}
    one = _iters(4, nel, precond)
    print(f"PCG iterations to 1e-10, {precond} pieces: two-level {two}, one-level at 4 slabs {one}")
    assert two[4] <= 1.2 * two[2]
    assert two[4] < 0.75 * one


def _simp_rank(rank, world, port, nel, rmin, out):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import fem
        from topogpu_b200.slab import Slab, SlabCoarse, SlabFilter, SlabPCG, all_dots, coarse_prolongation, \
            element_halo, slab_oc_filtered

        bc = fem.cantilever_bc(nel)
        bc.free_mask = lambda: _bc_free_mask(bc)
        slab = Slab.of(nel, rank, world, overlap=1)
        per = nel[1] * nel[2]
        ea, eb = slab.element_range(slab.e0, slab.e1)
        rho_g = np.random.default_rng(3).uniform(0.2, 0.9, int(np.prod(nel)))
        rho = torch.as_tensor(rho_g[ea:eb].copy())
        filt = SlabFilter(slab, rmin, dist)
        rho_f = filt.apply(rho)
        E_own = 1e-9 + (1 - 1e-9) * rho_f ** 3
        # the moduli the Schwarz pieces need (layers x_lo .. x_hi) from the halo
        hh = max(slab.e0 - slab.x_lo, slab.x_hi - slab.e1)
        E_ext = element_halo(E_own, slab, hh, dist).numpy()
        E_glob = np.zeros(int(np.prod(nel)))
        lo = max(slab.e0 - hh, 0)
        E_glob[lo * per:lo * per + len(E_ext)] = E_ext
        ops = OracleSlabOps(slab, bc, E_glob, "exact")
        P0 = coarse_prolongation(nel, _bc_free_mask(bc), 1)
        a, b = slab.dof_range()
        P = torch.as_tensor(P0[a:b].toarray())
        coarse = SlabCoarse(slab, P, SlabCoarse.galerkin(slab, P, ops.matvec, dist), dist)
        pcg = SlabPCG(slab, ops, dist, coarse=coarse, balanced=True)
        F = torch.as_tensor((bc.F * _bc_free_mask(bc))[a:b].copy())
        u, it, rr, ok = pcg.solve(F, tol=1e-13, maxiter=400)
        (c,) = all_dots([(F, u)], pcg.w, dist, world)
        dc = torch.as_tensor(fem.sensitivity(u.numpy(), rho_f.numpy(), slab.local_nel))
        dcd = filt.apply_transpose(dc)
        colsum = filt.apply_transpose(torch.ones_like(rho))
        rho_new, k = slab_oc_filtered(rho, dcd, colsum, colsum, 0.3, 0.2, slab, dist)
        out[rank] = {"rho_new": rho_new.numpy(), "rho_f": rho_f.numpy(), "c": c, "evals": k, "ok": ok,
                     "ea": ea, "eb": eb}
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,rmin", [(2, 2.0), (3, 1.5), (4, 2.3)])
def test_slab_simp_step_matches_single_process(world, rmin):
    """One filtered SIMP iteration on slabs (distributed filter with a halo
    of floor(rmin) element layers, two-level slab PCG, local sensitivities,
    H^T chain, filtered OC with the volume all-reduced per bisection step)
    against the undivided oracle step with a direct solve: filtered density
    to round-off, compliance and the new density to 1e-8, same number of OC
    evaluations."""
    from oracle import design, fem

    nel = (16, 4, 4)
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_simp_rank, args=(world, port, nel, rmin, out), nprocs=world, join=True)
        res = dict(out)
    bc = fem.cantilever_bc(nel)
    rho = np.random.default_rng(3).uniform(0.2, 0.9, int(np.prod(nel)))
    H = design.filter_matrix(nel, rmin)
    rf = H @ rho
    E = fem.simp_modulus(rf)
    U = fem.direct_solve(E, nel, bc)
    c_ref = float(bc.F @ U)
    dc = fem.sensitivity(U, rf, nel)
    dv = H.T @ np.ones(len(rho))
    ref, k_ref = design.oc_update_filtered(rho, H.T @ dc, dv, 0.3, 0.2, H)
    for r in res.values():
        assert r["ok"]
        np.testing.assert_allclose(r["rho_f"], rf[r["ea"]:r["eb"]], rtol=1e-13, atol=1e-15)
        assert abs(r["c"] - c_ref) / c_ref < 1e-8
        assert r["evals"] == k_ref
        np.testing.assert_allclose(r["rho_new"], ref[r["ea"]:r["eb"]], rtol=1e-8, atol=1e-10)
