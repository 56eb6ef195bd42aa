"""Many small meshes of uneven sizes, solved concurrently on one GPU.

``BatchSolver(meshes)`` keeps one ``StateSolver`` per mesh (its own GMG
hierarchy and its own CUDA-graph-captured PCG iteration, reused from solve to
solve) and runs the state solves from a pool of worker threads, each on its
own CUDA stream. The ctypes calls into libtopo_b200.so release the GIL, so the
kernels of different meshes overlap on the GPU and the host-side polling of
one solve hides behind the kernels of the others.

``autotune`` picks the worker count and the level-0 operator variant (tcgen05
or CUDA cores, same BF16 inputs and FP32 accumulation) by timing one round of
solves per candidate; the choice is cached under the batch's size signature
and reused by ``solve``.

The reference solves one mesh at a time; this is the batched form of its
SolverV4.solve (src/gpu_fem/solver_v4.py:147-269) for many independent
problems.
"""

from __future__ import annotations

import statistics
import threading
import time
from dataclasses import dataclass, field

import torch

from .bc import cantilever_edge_load
from .state import StateSolver


@dataclass
class BatchResult:
    compliance: list
    iterations: list
    latency_ms: list
    wall_s: float
    converged: list
    config: dict = field(default_factory=dict)

    @property
    def solves_per_s(self) -> float:
        return len(self.compliance) / self.wall_s

    def latency_percentile(self, q: float) -> float:
        xs = sorted(self.latency_ms)
        k = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
        return xs[k]


class BatchSolver:
    """State solves for a list of cantilever meshes ``[(nelx, nely, nelz), ...]``."""

    _tuned: dict = {}

    def __init__(self, meshes, *, precision="mixed", n_levels=4, tol=1e-5, maxiter=800, fine_degree=2,
                 loads=None, device=None):
        self.meshes = [tuple(int(v) for v in m) for m in meshes]
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.states = []
        for j, nel in enumerate(self.meshes):
            mask, F = loads[j] if loads is not None else cantilever_edge_load(nel)
            levels = max(1, min(n_levels, _max_levels(nel)))
            self.states.append(StateSolver(nel, mask, F, n_levels=levels, precision=precision, tol=tol,
                                           maxiter=maxiter, fine_degree=fine_degree, device=self.device))
        self.precision = precision

    def signature(self):
        return (self.precision, tuple(sorted(self.meshes)))

    def _set_tc(self, on: bool):
        for st in self.states:
            st.ctx.set_tensor_cores(on)

    def solve(self, rhos, *, workers=None, tensor_cores=None, penal=3.0, cold=True) -> BatchResult:
        """One state solve per mesh. cold=True starts every PCG from zero (a
        batch of new problems); cold=False warm-starts from each mesh's last
        solution (a design loop over the same meshes)."""
        tuned = BatchSolver._tuned.get(self.signature(), {})
        workers = workers or tuned.get("workers", 4)
        tc = tuned.get("tensor_cores", True) if tensor_cores is None else tensor_cores
        self._set_tc(tc)
        n = len(self.states)
        rhos = [torch.as_tensor(r, dtype=torch.float64, device=self.device) for r in rhos]
        order = sorted(range(n), key=lambda j: -self.states[j].ctx.n_elem)  # largest first
        comp, iters, lat, conv = [0.0] * n, [0] * n, [0.0] * n, [False] * n
        lock = threading.Lock()
        nxt = [0]
        errors = []

        def work():
            stream = torch.cuda.Stream(self.device)
            try:
                with torch.cuda.device(self.device), torch.cuda.stream(stream):
                    while True:
                        with lock:
                            if nxt[0] >= n:
                                return
                            j = order[nxt[0]]
                            nxt[0] += 1
                        t0 = time.perf_counter()
                        if cold:
                            self.states[j].reset_warm_start()
                        c, _ = self.states[j].solve(rhos[j], penal)
                        stream.synchronize()
                        lat[j] = (time.perf_counter() - t0) * 1e3
                        comp[j], iters[j], conv[j] = c, self.states[j].last_cg_iters, self.states[j].last_converged
            except BaseException as e:  # re-raised in the caller
                errors.append(e)

        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        threads = [threading.Thread(target=work) for _ in range(max(1, int(workers)))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        torch.cuda.synchronize(self.device)
        wall = time.perf_counter() - t0
        if errors:
            raise errors[0]
        return BatchResult(comp, iters, lat, wall, conv, {"workers": int(workers), "tensor_cores": bool(tc)})

    def autotune(self, rhos, candidates=((1, True), (2, True), (4, True), (8, True), (4, False), (8, False))):
        """Time one round per (workers, tensor_cores) candidate; keep the fastest."""
        best = None
        trials = []
        for w, tc in candidates:
            res = self.solve(rhos, workers=w, tensor_cores=tc)
            trials.append({"workers": w, "tensor_cores": tc, "solves_per_s": res.solves_per_s})
            if best is None or res.solves_per_s > best[0]:
                best = (res.solves_per_s, w, tc)
        BatchSolver._tuned[self.signature()] = {"workers": best[1], "tensor_cores": best[2]}
        return {"choice": BatchSolver._tuned[self.signature()], "trials": trials}

    def close(self):
        for st in self.states:
            st.close()


def _max_levels(nel) -> int:
    """Levels until a dimension would stop halving (factor-2 coarsening keeps >= 1 element)."""
    k, dims = 1, list(nel)
    while min(dims) >= 2 and k < 8:
        dims = [max(1, d // 2) for d in dims]
        k += 1
    return k


def config4b_meshes(count=64, seed=0):
    """Seeded uneven cantilevers: nelx ~ U{16..64}, nely = nelx // 2, nelz ~ U{8..32}."""
    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nx = int(rng.integers(16, 65))
        out.append((nx, nx // 2, int(rng.integers(8, 33))))
    return out


def summarize(res: BatchResult) -> dict:
    return {"solves": len(res.compliance), "solves_per_s": res.solves_per_s,
            "latency_ms_p50": res.latency_percentile(50), "latency_ms_p99": res.latency_percentile(99),
            "mean_pcg_iters": statistics.mean(res.iterations), "all_converged": all(res.converged), **res.config}
