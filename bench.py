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


def ku_micro(reps: int = 100, pairs: int = 8):
    """Level-0 K.u on the 192x96x48 grid: FP64, FP32 and BF16-input, with
    rotating buffers (> L2). Returns per-precision GDoF/s, bytes and times."""
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
    for name, dt in (("fp64", torch.float64), ("fp32", torch.float32), ("bf16", torch.bfloat16)):
        Edt = torch.float64 if dt == torch.float64 else torch.float32
        E = E64.to(Edt)
        us = [(torch.randn(ndof, generator=g) * mask.astype(np.float32)).to(dev).to(dt) for _ in range(pairs)]
        ys = [torch.empty(ndof, dtype=Edt, device=dev) for _ in range(pairs)]
        for k in range(3):
            ctx.matvec(us[k % pairs], E, out=ys[k % pairs])
        torch.cuda.synchronize()
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
                     "gflops": 1152 * ne / (ms * 1e-3) / 1e9, "launches": int(ctx._lib.topo_launch_count() - n0)}
    ctx.close()
    return out


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


def cpu_baseline(sample_nel=(48, 24, 24), steps=3):
    """The CPU oracle (restated reference SolverV4 GMG-PCG with its default
    FP32 smoother, filtered OC) on a reduced cantilever, scaled to 1M
    elements by element count."""
    from oracle import fem, simp

    bc = fem.cantilever_bc(sample_nel)
    s = simp.FilteredSIMP(sample_nel, bc, 0.30, 2.0, move=0.2, n_levels=4, fine_prec="fp32", fine_degree=3,
                          tol=1e-5, maxiter=800)
    t0 = time.perf_counter()
    its = []
    for _ in range(steps):
        s.step()
        its.append(s.state.last_iters)
    dt = time.perf_counter() - t0
    ne = int(np.prod(sample_nel))
    scale = ne / float(np.prod(NEL))
    rate = steps / dt * scale
    cores = len(os.sched_getaffinity(0))
    return {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": (f"{steps} filtered SIMP iterations of the oracle (reference SolverV4 GMG-PCG, FP32 smoother, "
                       f"deg 3, 4 levels, rtol 1e-5; PCG its {its}) on the {'x'.join(map(str, sample_nel))} "
                       f"cantilever ({ne} elements) in {dt:.1f} s on {cores} host cores (NumPy/SciPy threads), "
                       f"rate scaled to 1,024,000 elements by element count")}


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
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", str(len(os.sched_getaffinity(0))))
    from oracle import fem, simp

    nel = (48, 24, 24)
    bc = fem.cantilever_bc(nel)
    s = simp.FilteredSIMP(nel, bc, 0.30, 2.0, move=0.2, n_levels=4, fine_prec="fp32", fine_degree=3, tol=1e-5,
                          maxiter=800)
    for _ in range(args.warmup):
        s.step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        s.step()
        times.append(time.perf_counter() - t0)
    scale = float(np.prod(nel)) / float(np.prod(NEL))
    ms = statistics.mean(times) * 1e3 / scale
    value = 1e3 / ms
    cores = len(os.sched_getaffinity(0))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "cantilever 160x80x80 (1,024,000 hex) filtered SIMP, GMG-PCG rtol 1e-5",
                       "sample": "48x24x24 (27,648 hex) per step, rate scaled by element count",
                       "parallelism": "host CPU"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "one SIMP iteration of the CPU oracle (restated reference SolverV4 "
                                       "GMG-PCG, FP32 smoother) on 48x24x24 per step, scaled by element count"},
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
        print(json.dumps({"ku": ku_micro(args.micro_reps)}))
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
    roof = {"kernel": "tc::k_level0_tc<float, Store> (level-0 K.u, tcgen05 BF16 input, FP32 accumulate in TMEM)",
            "workload": "192x96x48 hex8 (2,751,987 DoF), 8 rotating (u,y) pairs", "bound": "hbm",
            "achieved": b["gbs"], "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": b["gbs"] / pk["hbm_gbs"],
            "traffic": None, "peak_source": pk["source"], "bytes_per_launch": b["bytes"],
            "launch_ms": b["ms"]}
    tr = ROOT / "profiles" / "k_level0_tc_192x96x48_traffic.json"
    if tr.exists():
        roof["traffic"] = json.loads(tr.read_text()).get("bytes_per_launch")

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
            "ku": {k: {"gdof_s": v["gdof_s"], "gbs": v["gbs"], "ms": v["ms"], "gflops": v["gflops"]}
                   for k, v in micro.items()},
            "roofline": roof,
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
