"""GPU parts of the x-slab decomposition (topogpu_b200.slab.CudaSlabOps).

One GPU: the slabs of two ranks are evaluated one after the other in this
process and their interface planes are summed here, so nothing waits on
another rank. Checks the slab contexts (local K u, the extended slab with
its fixed outer planes, the plane offsets) against the oracle on the same
inputs: K u to FP64 round-off, the Schwarz piece (a reference-smoother
V-cycle) to 1e-10 against the oracle V-cycle of the same extended problem,
and a one-rank SlabPCG to the direct solution.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import fem, gmg

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _mask(bc):
    m = np.zeros(bc.ndof, dtype=np.uint8)
    m[bc.free] = 1
    return m


def test_two_slabs_match_global_operator_and_schwarz_pieces(cuda_dev):
    from topogpu_b200.slab import CudaSlabOps, Slab

    nel = (16, 4, 4)
    bc = fem.cantilever_bc(nel)
    mask = _mask(bc)
    E = fem.simp_modulus(np.random.default_rng(3).uniform(0.1, 1.0, int(np.prod(nel))))
    Et = torch.as_tensor(E, device=DEV)
    slabs = [Slab.of(nel, r, 2) for r in range(2)]
    ops = [CudaSlabOps(s, mask, Et, n_levels=2, smoother="reference") for s in slabs]
    u = np.random.default_rng(4).standard_normal(bc.ndof) * mask
    ys = []
    for s, o in zip(slabs, ops):
        a, b = s.dof_range()
        ys.append(o.matvec(torch.as_tensor(u[a:b].copy(), device=DEV)).cpu().numpy())
    pd = slabs[0].plane_dofs
    iface = ys[0][-pd:] + ys[1][:pd]
    ys[0][-pd:] = iface
    ys[1][:pd] = iface
    yg = fem.matvec_full(u, E, nel) * mask
    for s, y in zip(slabs, ys):
        a, b = s.dof_range()
        assert np.abs(y - yg[a:b]).max() <= 1e-12 * np.abs(yg).max()
    for s, o in zip(slabs, ops):
        a, b = s.dof_range()
        z = o.precondition(torch.as_tensor(u[a:b].copy(), device=DEV)).cpu().numpy()
        m_ext = s.ext_free_mask(mask)
        free_ext = np.flatnonzero(m_ext)
        ea, eb = s.element_range(s.x_lo, s.x_hi)
        h = gmg.GMG(s.ext_nel, free_ext, n_levels=2, fine_prec="fp64", fine_degree=2).setup(E[ea:eb])
        ext = np.zeros(len(m_ext))
        off = s.ext_offset()
        ext[off:off + s.ndof] = u[a:b]
        zr = np.zeros(len(m_ext))
        zr[free_ext] = h.apply(ext[free_ext])
        zr = zr[off:off + s.ndof]
        assert np.linalg.norm(z - zr) / np.linalg.norm(zr) < 1e-10


def test_one_rank_slab_pcg_is_the_plain_solve(cuda_dev):
    import torch.distributed as dist

    from topogpu_b200.slab import CudaSlabOps, Slab, SlabPCG

    nel = (16, 8, 4)
    bc = fem.cantilever_bc(nel)
    mask = _mask(bc)
    E = fem.simp_modulus(np.random.default_rng(6).uniform(0.1, 1.0, int(np.prod(nel))))
    slab = Slab.of(nel, 0, 1)
    ops = CudaSlabOps(slab, mask, torch.as_tensor(E, device=DEV), n_levels=3)
    pcg = SlabPCG(slab, ops, dist, device=DEV)
    x, it, rr, ok = pcg.solve(torch.as_tensor(bc.F * mask, device=DEV), tol=1e-10, maxiter=300)
    U = fem.direct_solve(E, nel, bc)
    assert ok and rr < 1e-10 and it < 60
    assert np.abs(x.cpu().numpy() - U).max() < 1e-7 * np.abs(U).max()
