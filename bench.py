#!/usr/bin/env python
"""Benchmark: 1M-hex SIMP iterations/s (mixed vs plain FP32) and level-0 K.u roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (a "step" = one SIMP iteration, filter + state solve + sensitivity
+ filtered OC): the 160x80x80 hex8 cantilever (1,024,000 elements,
3,168,963 DoF), x=0 face clamped, unit -z load spread over the x=160, z=0
edge, volfrac 0.30, filter rmin 2.0, move 0.2, 4-level Galerkin GMG with
Chebyshev degree 3, FP32 outer PCG to rtol 1e-5 (<= 800 iterations).
Headline: mixed precision (BF16-input operators on levels 0-2, FP64 Cholesky
on level 3); the plain all-FP32 form runs beside it. Synthetic input, L2
flushed between steps. N>1 runs N independent replicas (the single mesh is
not sharded), so value = N x the slowest rank's rate.

The roofline object describes the dominant hot kernel named by the metric,
the level-0 BF16-input K.u, measured live here on the 192x96x48 operator
microbenchmark with 8 rotating (u, y) pairs (> L2).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "1M-hex SIMP iter/s @rtol1e-5, mixed vs plain FP32; K·u GDoF/s & %HBM roof"
UNIT = "SIMP iter/s"
NEL = (160, 80, 80)
MICRO_NEL = (192, 96, 48)
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def traffic_for(name: str):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
    a kernel from its committed ncu summary, used only while the sources that
    compile into that kernel (listed in the summary, with the build flags'
    file) are byte for byte the ones it was captured from, else None. The
    sources, not the library, are hashed: nvcc builds of the same source
    differ in embedded module identifiers."""
    import hashlib

    f = ROOT / "profiles" / f"{name}_traffic.json"
    if not f.exists():
        return None
    d = json.loads(f.read_text())
    srcs = d.get("sources")
    if not srcs or any(not (ROOT / p).exists() for p in srcs):
        return None
    h = hashlib.sha256()
    for p in srcs:
        h.update((ROOT / p).read_bytes())
    if d.get("src_sha256") != h.hexdigest():
        return None
    return d.get("bytes_per_launch")


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]), "source": "measured"}
    return {**FALLBACK_PEAKS, "source": "fallback"}


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = [r.split(",") for r in Path(self.path).read_text().splitlines() if r.count(",") >= 8]
        os.unlink(self.path)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def _rel_l2(a, b):
    a, b = a.double(), b.double()
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def ku_micro(reps: int = 100, pairs: int = 8):
    """Level-0 K.u on the 192x96x48 grid: FP64, FP32 and BF16-input, with
    rotating buffers (> L2). Returns per-precision GDoF/s, algorithmic bytes,
    times, launch counts and the relative L2 error of the FP32 and BF16
    operators against FP64 on the same u and E. Algorithmic bytes per launch:
    ndof*(s_u + s_y) + nelem*s_E (structured element map computed, vectors
    read or written once); the reference's 340 B/element model
    (experiments/paper4/run_experiments_e1_e10.py:659-660) is reported beside
    it, labelled as that model."""
    from topogpu_b200.bc import cantilever_edge_load
    from topogpu_b200.context import TopoContext

    dev = torch.device("cuda", torch.cuda.current_device())
    ctx = TopoContext(MICRO_NEL, n_levels=1, mode="fp32")
    mask, F = cantilever_edge_load(MICRO_NEL)
    mask_t = torch.tensor(mask, device=dev)
    ctx.set_problem(mask_t, torch.tensor(F, device=dev))
    g = torch.Generator(device="cpu").manual_seed(1)
    rho = torch.rand(ctx.n_elem, generator=g, dtype=torch.float64) * 0.999 + 0.001
    E64 = (1e-9 + (1 - 1e-9) * rho ** 3).to(dev)
    out = {}
    ndof, ne = ctx.ndof, ctx.n_elem
    base = [(torch.randn(ndof, generator=g, dtype=torch.float64) * torch.tensor(mask, dtype=torch.float64)).to(dev)
            for _ in range(pairs)]
    first = {}
    for name, dt in (("fp64", torch.float64), ("fp32", torch.float32), ("bf16", torch.bfloat16)):
        Edt = torch.float64 if dt == torch.float64 else torch.float32
        E = E64.to(Edt)
        us = [b.to(dt) for b in base]
        ys = [torch.empty(ndof, dtype=Edt, device=dev) for _ in range(pairs)]
        for k in range(3):
            ctx.matvec(us[k % pairs], E, out=ys[k % pairs])
        torch.cuda.synchronize()
        first[name] = ctx.matvec(us[0], E).clone()
        n0 = ctx._lib.topo_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(reps):
            ctx.matvec(us[k % pairs], E, out=ys[k % pairs])
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        s_u = {"fp64": 8, "fp32": 4, "bf16": 2}[name]
        s_y = 8 if name == "fp64" else 4
        byts = ndof * (s_u + s_y) + ne * (8 if name == "fp64" else 4)
        out[name] = {"ms": ms, "gdof_s": ndof / (ms * 1e-3) / 1e9, "bytes": byts, "gbs": byts / (ms * 1e-3) / 1e9,
                     "gflops": 1152 * ne / (ms * 1e-3) / 1e9,
                     "ref_model_gbs": 340.0 * ne / (ms * 1e-3) / 1e9,
                     "launches_per_apply": (ctx._lib.topo_launch_count() - n0) / reps}
    out["fp32"]["rel_l2_vs_fp64"] = _rel_l2(first["fp32"], first["fp64"])
    out["bf16"]["rel_l2_vs_fp64"] = _rel_l2(first["bf16"], first["fp64"])
    out["kernels"] = {"fp64": "k_level0_cc<double, Store> (CUDA cores, TMA-staged x-planes)",
                      "fp32": "k_level0_cc<float, Store> (CUDA cores, TMA-staged x-planes)",
                      "bf16": "k_level0_xs<bf16, Store> (tcgen05 node-pair tiles, BF16 u, TMA-staged x-planes)"}
    ctx.close()
    return out


def cheb_micro(reps: int = 30, sets: int = 3):
    """The Chebyshev step the mixed smoother runs on level 0, alone: the
    tensor-core K.u with FP32 u rounded to BF16 when staged and the fused
    epilogue r -= s K u; d = c1 u + c2 dinv r; x += ax d, on the 160x80x80
    SIMP mesh with `sets` rotating vector sets (> L2). Algorithmic bytes per
    launch: ndof*(4 u + 8 r + 4 dinv + 8 x + 4 d) + nelem*4 E."""
    from topogpu_b200.bc import cantilever_edge_load
    from topogpu_b200.context import TopoContext

    dev = torch.device("cuda", torch.cuda.current_device())
    ctx = TopoContext(NEL, n_levels=1, mode="mixed")
    mask, F = cantilever_edge_load(NEL)
    ctx.set_problem(torch.tensor(mask, device=dev), torch.tensor(F, device=dev))
    g = torch.Generator(device="cpu").manual_seed(2)
    rho = torch.rand(ctx.n_elem, generator=g, dtype=torch.float64) * 0.999 + 0.001
    E = (1e-9 + (1 - 1e-9) * rho ** 3).float().to(dev)
    m = torch.tensor(mask, dtype=torch.float32, device=dev)
    nd, ne = ctx.ndof, ctx.n_elem

    def vec():
        return torch.randn(nd, generator=g).to(dev) * m

    S = [dict(u=vec(), r=vec(), x=vec(), d=torch.zeros(nd, device=dev), dinv=(torch.rand(nd, generator=g).to(dev) + 0.1) * m)
         for _ in range(sets)]

    def run(k):
        v = S[k % sets]
        ctx.level0_apply(v["u"], E, "cheb", r=v["r"], x=v["x"], d_out=v["d"], dinv=v["dinv"], s=0.5, c1=0.3, c2=0.9,
                         ax=1.0, u_fp32_to_bf16=True)

    for k in range(3):
        run(k)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(reps):
        run(k)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    byts = nd * 28 + ne * 4
    ctx.close()
    return {"kernel": "k_level0_xs<float, ChebR> (tcgen05 node-pair tiles, FP32 u rounded to BF16, fused Chebyshev epilogue)",
            "workload": "160x80x80 hex8 (3,168,963 DoF), 3 rotating vector sets", "ms": ms, "bytes": byts,
            "gbs": byts / (ms * 1e-3) / 1e9, "gdof_s": nd / (ms * 1e-3) / 1e9}


def simp_steps(precision, steps, warmup, flush, rmin=2.0):
    """Time `steps` SIMP iterations after `warmup` untimed ones (device events)."""
    import topogpu_b200 as tg
    from topogpu_b200.solver import SIMPLoop

    p = tg.gallery.benchmark_cantilever(NEL, volfrac=0.30, filter_radius=rmin)
    solver = tg.SIMPSolver(backend="cuda", tol=1e-5, max_krylov=800, move=0.2, precision=precision, levels=4,
                           fine_degree=3, coarse_degree=2, use_filter=True)
    loop = SIMPLoop(solver, p)
    lib = loop.state.ctx._lib
    rows = []
    for _ in range(warmup):
        rows.append(loop.step(stats=False))
    times, launches, phases = [], 0, []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0 = lib.topo_launch_count()
        loop.state.timing = True
        e0.record()
        rows.append(loop.step(stats=False))
        e1.record()
        torch.cuda.synchronize()
        launches += int(lib.topo_launch_count() - n0)
        times.append(e0.elapsed_time(e1))
        phases.append(dict(loop.state.last_timing))
    info = loop.state.ctx.gmg_info()
    info["setup_phases_ms"] = loop.state.ctx.setup_phases()
    loop.close()
    keys = ("gmg_setup_ms", "cg_ms", "sensitivity_ms")
    breakdown = {k: statistics.mean(ph[k] for ph in phases) for k in keys} if phases and phases[0] else {}
    if breakdown:
        breakdown["design_update_ms"] = statistics.mean(times) - statistics.mean(ph["total_ms"] for ph in phases)
    return {"ms": times, "rows": rows, "launches": launches, "gmg": info, "breakdown": breakdown}


def e2e_steps(precision, steps, warmup, flush, rmin=2.0):
    """Same SIMP step through the public API with the density crossing the host
    boundary every step: pinned H2D of rho in, D2H of the new rho out."""
    import topogpu_b200 as tg
    from topogpu_b200.solver import SIMPLoop

    p = tg.gallery.benchmark_cantilever(NEL, volfrac=0.30, filter_radius=rmin)
    solver = tg.SIMPSolver(backend="cuda", tol=1e-5, max_krylov=800, move=0.2, precision=precision, levels=4,
                           fine_degree=3, coarse_degree=2, use_filter=True)
    loop = SIMPLoop(solver, p)
    n = loop.rho.numel()
    h_in = torch.full((n,), 0.30, dtype=torch.float64).pin_memory()
    h_out = torch.empty(n, dtype=torch.float64).pin_memory()
    for _ in range(warmup):
        loop.step_host(h_in, h_out)
        h_in.copy_(h_out)
    times = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        loop.step_host(h_in, h_out)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
        h_in.copy_(h_out)
    loop.close()
    return {"ms": times, "h2d": n * 8, "d2h": n * 8}


def fp64_compliance_check(rho_first=0.30, rmin=2.0):
    """Compliance of the first SIMP state in mixed and FP64 modes (same rho)."""
    import topogpu_b200 as tg

    out = {}
    p = tg.gallery.benchmark_cantilever(NEL, volfrac=0.30, filter_radius=rmin)
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-5)):
        s = tg.SIMPSolver(backend="cuda", tol=tol, max_krylov=800, precision=prec, levels=4, fine_degree=3)
        st = s.make_state_solver(p)
        rho = torch.full((st.ctx.n_elem,), rho_first, dtype=torch.float64, device=st.device)
        c, _ = st.solve(rho, 3.0)
        out[prec] = c
        st.close()
    return abs(out["mixed"] - out["fp64"]) / abs(out["fp64"])


# The CPU oracle's SIMP iteration at 160x80x80 takes minutes, so both CPU
# measurements time a sample mesh with 1/15.6 of its elements and carry the
# time linearly in the element count. Checked against a direct oracle run at
# 160x80x80 on 8 host cores: 162.8 s per iteration there (two iterations,
# PCG its 15 and 32) against 9.89 s x 15.625 = 154.5 s from this sample (PCG
# its 15 and 26). Fitted power laws over smaller pairs of meshes were further
# off (24x12x12 and 48x24x24: t ~ n^0.77, 46.9 s).
REF_SAMPLE = (64, 32, 32)


def _oracle_step_seconds(nel, steps):
    """Seconds per filtered SIMP iteration of the CPU oracle (the restated
    reference SolverV4 GMG-PCG: FP64 PCG, FP32 Chebyshev smoother, degree 3,
    4 levels, rtol 1e-5; filter rmin 2.0, move 0.2) on an nel cantilever,
    averaged over `steps` iterations from the uniform start."""
    from oracle import fem, simp

    bc = fem.cantilever_bc(nel)
    s = simp.FilteredSIMP(nel, bc, 0.30, 2.0, move=0.2, n_levels=4, fine_prec="fp32", fine_degree=3, tol=1e-5,
                          maxiter=800)
    t0 = time.perf_counter()
    its = []
    for _ in range(steps):
        s.step()
        its.append(s.state.last_iters)
    return (time.perf_counter() - t0) / steps, its


def scale_to_full(t_sample_s):
    """Seconds per 160x80x80 iteration from a REF_SAMPLE iteration (linear in elements)."""
    return t_sample_s * float(np.prod(NEL)) / float(np.prod(REF_SAMPLE))


def cpu_baseline(steps=2):
    """The CPU oracle's SIMP iteration rate at 160x80x80, carried linearly
    from `steps` iterations on the REF_SAMPLE mesh (a bounded sample)."""
    t, its = _oracle_step_seconds(REF_SAMPLE, steps)
    t_full = scale_to_full(t)
    cores = len(os.sched_getaffinity(0))
    return {"value": 1.0 / t_full, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": (f"{steps} filtered SIMP iterations of the CPU oracle (restated reference SolverV4 GMG-PCG, FP64 "
                       f"PCG, FP32 smoother deg 3, 4 levels, rtol 1e-5) on {'x'.join(map(str, REF_SAMPLE))} "
                       f"({int(np.prod(REF_SAMPLE))} hex, {t:.2f} s/it, PCG its {its}), carried to 1,024,000 hex "
                       f"linearly in the element count (checked on 8 cores against a direct 160x80x80 run: "
                       f"154.5 s predicted, 162.8 s measured); {cores} host cores (NumPy/SciPy threads)")}


def max_over_ranks(x: float, dist, device="cuda") -> float:
    """Max of a per-rank time over all ranks (the slowest rank sets the job time)."""
    if dist is None:
        return float(x)
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world: int, ms_per_step: float) -> float:
    """Whole-job SIMP iterations/s of `world` independent replicas."""
    return world * 1e3 / ms_per_step


def extras():
    """Multi-load block PCG (96x48x48, 8 seeded point loads) and 64 batched
    uneven cantilevers, both mixed precision at rtol 1e-5, device-synchronised
    wall time after a warm-up call."""
    from topogpu_b200.batch import BatchSolver, config4b_meshes, summarize
    from topogpu_b200.bc import cantilever_edge_load, face_point_loads
    from topogpu_b200.state import StateSolver

    out = {}
    nel = (96, 48, 48)
    mask, F = cantilever_edge_load(nel)
    rho = np.random.default_rng(31).uniform(0.05, 1.0, int(np.prod(nel)))
    B = face_point_loads(nel, 8, 32)
    st = StateSolver(nel, mask, F, n_levels=4, precision="mixed", tol=1e-5, maxiter=800, fine_degree=3)
    st.solve_block(rho, B)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    comps, _ = st.solve_block(rho, B)
    torch.cuda.synchronize()
    t_block = time.perf_counter() - t0
    it_block = st.last_cg_iters
    t0 = time.perf_counter()
    its = 0
    for j in range(8):
        x = torch.zeros(st.ctx.ndof, dtype=torch.float64, device="cuda")
        i1, _, _ = st.ctx.pcg(torch.tensor(B[j] * mask, device="cuda"), x, 1e-5, 800)
        its += i1
    torch.cuda.synchronize()
    t_single = time.perf_counter() - t0
    st.close()
    out["block_pcg_96x48x48_8loads"] = {"block_ms": t_block * 1e3, "block_iters": it_block,
                                        "single_ms_total": t_single * 1e3, "single_iters_total": its,
                                        "speedup": t_single / t_block}
    meshes = config4b_meshes(64, seed=0)
    rng = np.random.default_rng(41)
    rhos = [torch.tensor(rng.uniform(0.05, 1.0, int(np.prod(m))), dtype=torch.float64, device="cuda")
            for m in meshes]
    bs = BatchSolver(meshes, precision="mixed", tol=1e-5)
    tune = bs.autotune(rhos)
    res = bs.solve(rhos)
    out["batched_64_uneven_cantilevers"] = {**summarize(res), "autotune_trials": tune["trials"]}
    bs.close()
    return out


def reference_arm(args, rank):
    """The reference's algorithm on the host cores (the CPU oracle: the
    reference is Python on CuPy, which is not installed, so it cannot run
    on the GPU box itself). Each step is one SIMP iteration of the REF_SAMPLE
    mesh, carried to 160x80x80 linearly in the element count. The run
    restarts from the uniform density every two iterations (construction not
    timed), so every step is iteration 1 or 2: the regime in which the
    linear scaling was checked against a direct 160x80x80 run, and a bounded
    cost per step (later iterations of the oracle's FP32 smoother need many
    more PCG iterations on this mesh: 60 and 162 at iterations 3 and 4)."""
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", str(len(os.sched_getaffinity(0))))
    from oracle import fem, simp

    bc = fem.cantilever_bc(REF_SAMPLE)
    state = {"s": None, "k": 0}

    def one_iteration():
        if state["k"] % 2 == 0:
            state["s"] = simp.FilteredSIMP(REF_SAMPLE, bc, 0.30, 2.0, move=0.2, n_levels=4, fine_prec="fp32",
                                           fine_degree=3, tol=1e-5, maxiter=800)
        state["k"] += 1
        t0 = time.perf_counter()
        state["s"].step()
        return time.perf_counter() - t0, state["s"].state.last_iters

    for _ in range(args.warmup):
        one_iteration()
    times, its = [], []
    for _ in range(args.steps):
        t, it = one_iteration()
        times.append(t)
        its.append(it)
    ms = scale_to_full(statistics.mean(times)) * 1e3
    value = 1e3 / ms
    cores = len(os.sched_getaffinity(0))
    sample = (f"{args.steps} SIMP iterations of the CPU oracle (restated reference SolverV4 GMG-PCG: FP64 PCG, FP32 "
              f"Chebyshev smoother deg 3, 4 levels, rtol 1e-5, filter rmin 2.0) on {'x'.join(map(str, REF_SAMPLE))} "
              f"({int(np.prod(REF_SAMPLE))} hex), each iteration 1 or 2 of a run restarted from the uniform density "
              f"every two (PCG its {its}, {statistics.mean(times):.2f} s/it), carried to 1,024,000 hex linearly in "
              f"the element count (checked on 8 cores against a direct 160x80x80 run of iterations 1-2: 154.5 s "
              f"predicted, 162.8 s measured)")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "sample_ms_per_step": statistics.mean(times) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 PCG / f32 smoother", "data": "synthetic",
            "config": {"workload": "cantilever 160x80x80 (1,024,000 hex) filtered SIMP, GMG-PCG rtol 1e-5",
                       "sample": sample, "parallelism": "host CPU"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=9)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the multi-load and batched-mesh measurements")
    ap.add_argument("--micro-reps", type=int, default=100)
    ap.add_argument("--only-ku", action="store_true", help="run only the K.u microbenchmark (profiling)")
    ap.add_argument("--only-simp", action="store_true", help="run only the mixed SIMP steps (profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank)

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from topogpu_b200 import _lib

    lib = _lib.load()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    if args.only_ku:
        print(json.dumps({"ku": ku_micro(args.micro_reps), "cheb": cheb_micro()}))
        return 0
    if args.only_simp:
        r = simp_steps("mixed", args.steps, args.warmup, flush)
        print(json.dumps({"ms": r["ms"], "breakdown": r["breakdown"], "launches": r["launches"],
                          "pcg_iters": [x["outer_iters"] for x in r["rows"]]}))
        return 0
    micro = ku_micro(args.micro_reps)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    n0 = lib.topo_launch_count()
    mixed = simp_steps("mixed", args.steps, args.warmup, flush)
    launches = mixed["launches"]
    clk = clocks.stop()
    torch.cuda.synchronize()
    total_ms = max_over_ranks(sum(mixed["ms"]), dist)
    ms_step = total_ms / args.steps
    value = replica_rate(world, ms_step)
    fp32 = None if args.no_fp32 else simp_steps("fp32", args.steps, args.warmup, flush)
    e2e = e2e_steps("mixed", args.steps, args.warmup, flush)
    e2e_ms = max_over_ranks(sum(e2e["ms"]), dist)
    rel_err = fp64_compliance_check()
    del n0

    pk = peaks()
    b = micro["bf16"]
    roof = {"kernel": micro["kernels"]["bf16"] + ", level-0 K.u y = K(E) u",
            "workload": "192x96x48 hex8 (2,751,987 DoF), 8 rotating (u,y) pairs", "bound": "hbm",
            "achieved": b["gbs"], "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": b["gbs"] / pk["hbm_gbs"],
            "traffic": traffic_for("k_level0_xs_bf16_store_192x96x48"), "peak_source": pk["source"],
            "bytes_per_launch": b["bytes"], "launch_ms": b["ms"]}
    ch = cheb_micro()
    roof_cheb = {"kernel": ch["kernel"], "workload": ch["workload"], "bound": "hbm", "achieved": ch["gbs"],
                 "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": ch["gbs"] / pk["hbm_gbs"],
                 "traffic": traffic_for("k_level0_xs_float_cheb_160x80x80"), "peak_source": pk["source"],
                 "bytes_per_launch": ch["bytes"], "launch_ms": ch["ms"]}

    iters = [r["outer_iters"] for r in mixed["rows"][args.warmup:]]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16-in/fp32 (mixed)", "data": "synthetic",
            "config": {"workload": "cantilever 160x80x80 (1,024,000 hex, 3,168,963 DoF) filtered SIMP, rmin 2.0",
                       "solver": "4-level Galerkin GMG, Chebyshev deg 3, BF16 L0-L2, FP64 Cholesky L3, "
                                 "FP32 PCG rtol 1e-5",
                       "parallelism": f"replicas x{world}", "l2": "flushed between steps (512 MB write)"},
            "pcg_iters_per_step": iters,
            "step_breakdown_ms": mixed["breakdown"],
            "compliance_rel_err_vs_fp64": rel_err,
            "plain_fp32": None if fp32 is None else {
                "value": world * 1e3 / (sum(fp32["ms"]) / args.steps), "ms_per_step": sum(fp32["ms"]) / args.steps,
                "pcg_iters_per_step": [r["outer_iters"] for r in fp32["rows"][args.warmup:]],
                "step_breakdown_ms": fp32["breakdown"]},
            "ku": {k: v for k, v in micro.items()},
            "roofline": roof,
            "roofline_cheb_step": roof_cheb,
            "clocks": clk,
            "gpu_launches": launches,
            "e2e": {"value": replica_rate(world, e2e_ms / args.steps), "unit": UNIT,
                    "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]},
            "gmg": mixed["gmg"]}
    if fp32 is not None:
        line["mixed_speedup_vs_fp32"] = line["plain_fp32"]["ms_per_step"] / ms_step
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if world == 1 and not args.no_extras:
        line["extras"] = extras()
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
