"""The range-checked library (built with TOPO_DEBUG_BOUNDS) on a whole
mixed-precision state solve, the level-0 operator in every precision, the
filter and the sensitivity: no gather/scatter index goes out of range, and
the results are the normal build's (compliance against the oracle to 1e-4).
Runs in a child process, since the library variant is chosen at load."""

from __future__ import annotations

import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import ctypes, numpy as np, torch
from oracle import fem
from topogpu_b200 import _lib
from topogpu_b200.context import TopoContext
from topogpu_b200.state import StateSolver
assert _lib.lib_path().name == "libtopo_b200_dbg.so"
lib = _lib.load()
nel = (24, 12, 10)
bc = fem.cantilever_bc(nel)
mask = np.zeros(bc.ndof, dtype=np.uint8); mask[bc.free] = 1
rho = np.random.default_rng(2).uniform(0.1, 1.0, int(np.prod(nel)))
st = StateSolver(nel, mask, bc.F, n_levels=3, precision="mixed", fine_degree=3, tol=1e-8, maxiter=300)
c, dc = st.solve(torch.tensor(rho, device="cuda"), 3.0)
u_ref = fem.direct_solve(fem.simp_modulus(rho), nel, bc)
c_ref = float(bc.F @ u_ref)
assert abs(c - c_ref) / c_ref < 1e-4, (c, c_ref)
ctx = TopoContext(nel, n_levels=1, mode="fp64")
ctx.set_problem(torch.tensor(mask, device="cuda"), torch.tensor(bc.F, device="cuda"))
E = torch.tensor(fem.simp_modulus(rho), device="cuda")
u = torch.tensor(u_ref, device="cuda")
for dt in (torch.float64, torch.float32, torch.bfloat16):
    ctx.matvec(u.to(dt), E.to(torch.float64 if dt == torch.float64 else torch.float32))
ctx.filter(2.0, torch.tensor(rho, device="cuda"))
ctx.filter(2.0, torch.tensor(rho, device="cuda"), transpose=True)
ctx.sensitivity(u, torch.tensor(rho, device="cuda"))
torch.cuda.synchronize()
t = ctypes.c_int(-1)
rc = lib.topo_debug_bounds(ctypes.byref(t))
print("bounds", rc, t.value)
assert rc == 0 and t.value == 0
"""


def test_range_checked_build_runs_clean(cuda_dev):
    from topogpu_b200 import build

    build.build(debug_bounds=True)
    env = {**os.environ, "TOPO_B200_LIB": "dbg", "PYTHONPATH": str(ROOT)}
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "bounds 0 0" in r.stdout
