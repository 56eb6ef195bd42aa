"""Tensor-core level-0 K.u (BF16 inputs, FP32 accumulation) and its fused
epilogues against the oracle.

The oracle emulates the kernel's arithmetic (u and KE rounded to BF16 with
round-to-nearest-even, element products formed exactly, the element vector
rounded to FP32 and scaled by E in FP32, then summed; the semantics of
fused_matvec_bf16 in src/gpu_fem/cuda_fused_matvec.py:112-246). The kernel
sums in FP32 in another order, so every comparison allows FP32 rounding:
relative L2 error below 1e-5 for the operator and each updated vector, fixed
DoFs exactly zero. Meshes cover the 192x96x48 microbenchmark and the
160x80x80 SIMP mesh (many CTAs, window restarts, node planes split between
CTAs), ragged windows in y, z extents that end exactly on a tile (the last
pair's thread finishes the top node) and ones that do not, and single-window
meshes. Every call goes through the C ABI (topo_level0_apply / topo_matvec).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import fem

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
TOL = 1e-5

MESHES = [(7, 5, 3), (24, 12, 6), (17, 8, 9), (33, 17, 40), (10, 31, 16), (12, 9, 80), (5, 46, 33)]
LARGE = [(192, 96, 48), (160, 80, 80)]


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _setup(nel, seed):
    from topogpu_b200.context import TopoContext

    bc = fem.cantilever_bc(nel)
    mask = np.zeros(bc.ndof, dtype=np.uint8)
    mask[bc.free] = 1
    ctx = TopoContext(nel, n_levels=1, mode="mixed")
    ctx.set_problem(torch.tensor(mask, device=DEV), torch.tensor(bc.F, device=DEV))
    rng = np.random.default_rng(seed)
    n = int(np.prod(nel))
    E = fem.simp_modulus(rng.uniform(0.001, 1.0, n)).astype(np.float32)
    u = rng.standard_normal(bc.ndof).astype(np.float32) * mask
    return ctx, bc, mask, E, u, rng


def _emu(u, E, nel, mask):
    y = fem.matvec_full(fem.bf16_round(u), E, nel, "bf16").astype(np.float64)
    y[mask == 0] = 0.0
    return y


def _t(a, dt=torch.float32):
    return torch.tensor(np.asarray(a), dtype=dt, device=DEV)


@pytest.mark.parametrize("nel", MESHES + LARGE)
def test_store_bf16_input_matches_emulation(cuda_dev, nel):
    ctx, bc, mask, E, u, _ = _setup(nel, 1)
    ub = _t(u).to(torch.bfloat16)
    y1 = ctx.level0_apply(ub, _t(E), "store").cpu().numpy()
    y2 = ctx.matvec(ub, _t(E)).cpu().numpy()
    ref = _emu(u, E, nel, mask)
    assert _rel(y1, ref) < TOL
    assert np.all(y1[mask == 0] == 0.0)
    # the kernel is deterministic (owner-computes, fixed summation order)
    assert np.array_equal(y1, y2)
    # exact linearity in powers of two: BF16 rounding commutes with scaling by 2
    y4 = ctx.level0_apply(_t(4.0 * u).to(torch.bfloat16), _t(E), "store").cpu().numpy()
    assert np.array_equal(y4, 4.0 * y1)
    ctx.close()


@pytest.mark.parametrize("nel", MESHES + LARGE)
def test_chebyshev_step_fp32_input_matches_oracle(cuda_dev, nel):
    """The smoother's form: u (the previous direction) FP32, rounded to BF16
    for the product but used at FP32 in d_out = c1 u + c2 dinv r."""
    ctx, bc, mask, E, u, rng = _setup(nel, 2)
    nd = bc.ndof
    r = rng.standard_normal(nd).astype(np.float32) * mask
    x = rng.standard_normal(nd).astype(np.float32)
    dinv = (rng.uniform(0.1, 1.0, nd) * mask).astype(np.float32)
    s, c1, c2, ax = 0.7, 0.3, 1.1, 0.9
    rt, xt, dt = _t(r), _t(x), torch.zeros(nd, dtype=torch.float32, device=DEV)
    ctx.level0_apply(_t(u), _t(E), "cheb", r=rt, x=xt, d_out=dt, dinv=_t(dinv), s=s, c1=c1, c2=c2, ax=ax,
                     u_fp32_to_bf16=True)
    w = _emu(u, E, nel, mask)
    fr = mask != 0
    r_ref = np.where(fr, r - s * w, 0.0)
    d_ref = np.where(fr, c1 * u.astype(np.float64) + c2 * dinv * r_ref, 0.0)
    x_ref = np.where(fr, x + ax * d_ref, x)
    got_r, got_d, got_x = rt.cpu().numpy(), dt.cpu().numpy(), xt.cpu().numpy()
    assert _rel(got_r, r_ref) < TOL
    assert _rel(got_d, d_ref) < TOL
    assert _rel(got_x, x_ref) < TOL
    assert np.all(got_r[~fr] == 0.0) and np.all(got_d[~fr] == 0.0)
    assert np.array_equal(got_x[~fr], x[~fr])
    ctx.close()


@pytest.mark.parametrize("nel", [(17, 8, 9), (33, 17, 40), (192, 96, 48)])
def test_residual_and_update_epilogues(cuda_dev, nel):
    ctx, bc, mask, E, u, rng = _setup(nel, 3)
    nd = bc.ndof
    b = rng.standard_normal(nd).astype(np.float32)
    r = rng.standard_normal(nd).astype(np.float32) * mask
    w = _emu(u, E, nel, mask)
    fr = mask != 0
    for uin, f32 in ((_t(u), True), (_t(u).to(torch.bfloat16), False)):
        y = ctx.level0_apply(uin, _t(E), "residual", b=_t(b), u_fp32_to_bf16=f32).cpu().numpy()
        assert _rel(y, np.where(fr, b - w, 0.0)) < TOL
        rt = _t(r)
        ctx.level0_apply(uin, _t(E), "rupd", r=rt, s=0.45, u_fp32_to_bf16=f32)
        assert _rel(rt.cpu().numpy(), np.where(fr, r - 0.45 * w, 0.0)) < TOL
    ctx.close()


def test_bf16_operator_close_to_fp64(cuda_dev):
    """BF16 inputs cost about three significant digits against the FP64
    operator (reported as rel_l2_vs_fp64 by the benchmark)."""
    nel = (48, 24, 24)
    ctx, bc, mask, E, u, _ = _setup(nel, 4)
    y64 = ctx.matvec(_t(u, torch.float64), _t(E, torch.float64)).cpu().numpy()
    yb = ctx.level0_apply(_t(u).to(torch.bfloat16), _t(E), "store").cpu().numpy()
    err = _rel(yb, y64)
    assert 1e-4 < err < 2e-2
    ctx.close()
