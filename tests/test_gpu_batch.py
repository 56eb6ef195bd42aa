"""Configuration 4b: 64 seeded cantilevers of uneven sizes (nelx ~ U{16..64},
nely = nelx // 2, nelz ~ U{8..32}) solved concurrently; every compliance is
checked against a one-at-a-time FP64 solve of the same mesh."""

import numpy as np
import pytest
import torch

from topogpu_b200.batch import BatchSolver, config4b_meshes, summarize


def _rhos(meshes, seed=41):
    rng = np.random.default_rng(seed)
    return [torch.tensor(rng.uniform(0.05, 1.0, int(np.prod(m))), dtype=torch.float64, device="cuda") for m in meshes]


@pytest.mark.gpu
def test_batched_uneven_meshes_match_single_fp64(cuda_dev):
    meshes = config4b_meshes(64, seed=0)
    assert any(m[2] % 2 for m in meshes)  # odd dimensions occur
    rhos = _rhos(meshes)
    bs = BatchSolver(meshes, precision="mixed", tol=1e-5)
    tune = bs.autotune(rhos)
    res = bs.solve(rhos)
    s = summarize(res)
    print("64 uneven meshes, autotune:", tune["choice"], "->", {k: (round(v, 2) if isinstance(v, float) else v)
                                                          for k, v in s.items()})
    assert s["all_converged"] and s["mean_pcg_iters"] > 0
    ref = BatchSolver(meshes, precision="fp64", tol=1e-10)
    r64 = ref.solve(rhos, workers=1)
    assert all(r64.converged)
    rel = np.abs(np.array(res.compliance) - np.array(r64.compliance)) / np.abs(np.array(r64.compliance))
    print(f"max compliance rel err mixed vs fp64: {rel.max():.2e}")
    assert rel.max() < 1e-4
    bs.close()
    ref.close()
