"""topo_oc_noalloc: the OC update for callers that cannot allocate device memory.

Callers whose device memory belongs to their own pool (a framework's caching
allocator, a Go or JVM runtime), or whose loop cannot afford the device-wide
synchronisation of cudaMalloc/cudaFree, use this entry point: it works in a
static scratch array inside the library instead of allocating. These tests
call it through the C ABI and check it against the context-based topo_oc,
bit for bit (the tolerance of the OC tests), on two calls in a row. The file
is named to be collected last and needs no state from the other tests.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import load_golden


def _noalloc(lib, rho, dc, volfrac, move, rho_min=1e-3):
    import torch

    out = torch.empty_like(rho)
    ev = C.c_int(0)
    rc = lib.topo_oc_noalloc(rho.data_ptr(), dc.data_ptr(), rho.numel(), float(volfrac), float(move),
                             float(rho_min), out.data_ptr(), C.byref(ev), torch.cuda.current_stream().cuda_stream)
    return rc, out, ev.value


def test_no_alloc_rejects_sizes_beyond_its_scratch():
    """The size check comes before any device access (runs without a GPU)."""
    from topogpu_b200 import _lib

    lib = _lib.load()
    ev = C.c_int(0)
    rc = lib.topo_oc_noalloc(None, None, 8_388_609, 0.3, 0.2, 1e-3, None, C.byref(ev), None)
    assert rc < 0
    assert "8388608" in _lib.last_error(None)
    assert lib.topo_oc_noalloc(None, None, 0, 0.3, 0.2, 1e-3, None, C.byref(ev), None) < 0


@pytest.mark.gpu
def test_no_alloc_oc_matches_context_oc_twice(cuda_dev):
    import torch

    from oracle import design
    from topogpu_b200 import _lib
    from topogpu_b200.context import TopoContext

    lib = _lib.load()
    g = load_golden("oc")
    rng = np.random.default_rng(12)
    n_big = 300_000
    # the reference's three OC fixtures, then a 300,000-element seeded case
    cases = [(g[f"rho_{k}"], g[f"dc_{k}"], float(g[f"vf_{k}"]), float(g[f"move_{k}"]), g[f"out_{k}"]) for k in range(3)]
    cases.append((rng.uniform(0.001, 1.0, n_big), -rng.gamma(1.0, 1.0, n_big) * 10.0 ** rng.uniform(-4, 1, n_big), 0.3,
                  0.2, None))
    for rho_np, dc_np, vf, mv, want in cases:
        rho = torch.tensor(rho_np, dtype=torch.float64, device=cuda_dev)
        dc = torch.tensor(dc_np, dtype=torch.float64, device=cuda_dev)
        ctx = TopoContext((rho.numel(), 1, 1), n_levels=1, mode="fp64")
        ref, ev_ref = ctx.oc(rho, dc, vf, mv)
        _, ev_oracle = design.oc_update(rho_np, dc_np, vf, mv)
        for _ in range(2):  # two calls in a row share (and must clear) the static scratch
            rc, out, ev = _noalloc(lib, rho, dc, vf, mv)
            assert rc == 0, _lib.last_error(None)
            assert torch.equal(out, ref)
            assert ev == ev_ref == ev_oracle
            if want is not None:
                assert np.array_equal(out.cpu().numpy(), want)
        ctx.close()


@pytest.mark.gpu
def test_no_alloc_oc_at_its_size_limit(cuda_dev):
    """n = 8,388,608 fills every partial-sum slot of the static scratch (the
    slots just below the bisection state); the result must equal the
    oracle's update bit for bit, twice in a row."""
    import torch

    from oracle import design
    from topogpu_b200 import _lib

    lib = _lib.load()
    n = 8_388_608
    rng = np.random.default_rng(21)
    rho_np = rng.uniform(0.001, 1.0, n)
    dc_np = -rng.gamma(1.0, 1.0, n) * 10.0 ** rng.uniform(-4, 1, n)
    want, ev_want = design.oc_update(rho_np, dc_np, 0.4, 0.2)
    rho = torch.tensor(rho_np, dtype=torch.float64, device=cuda_dev)
    dc = torch.tensor(dc_np, dtype=torch.float64, device=cuda_dev)
    for _ in range(2):
        rc, out, ev = _noalloc(lib, rho, dc, 0.4, 0.2)
        assert rc == 0, _lib.last_error(None)
        assert ev == ev_want
        assert np.array_equal(out.cpu().numpy(), want)
