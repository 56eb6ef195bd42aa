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

    from topogpu_b200 import _lib
    from topogpu_b200.context import TopoContext

    lib = _lib.load()
    g = load_golden("oc")
    rng = np.random.default_rng(12)
    n_big = 300_000
    cases = [(g["rho_0"], g["dc_0"], float(g["vf_0"]), float(g["move_0"])),
             (rng.uniform(0.001, 1.0, n_big), -rng.gamma(1.0, 1.0, n_big) * 10.0 ** rng.uniform(-4, 1, n_big), 0.3,
              0.2)]
    for rho_np, dc_np, vf, mv in cases:
        rho = torch.tensor(rho_np, dtype=torch.float64, device=cuda_dev)
        dc = torch.tensor(dc_np, dtype=torch.float64, device=cuda_dev)
        ctx = TopoContext((rho.numel(), 1, 1), n_levels=1, mode="fp64")
        ref, ev_ref = ctx.oc(rho, dc, vf, mv)
        for _ in range(2):  # two calls in a row share (and must clear) the static scratch
            rc, out, ev = _noalloc(lib, rho, dc, vf, mv)
            assert rc == 0, _lib.last_error(None)
            assert torch.equal(out, ref)
            assert ev == ev_ref
        ctx.close()
