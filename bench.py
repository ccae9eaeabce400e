"""Benchmark of the supernodal Cholesky factor + solve hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one GPU): 3D 7-point Laplacian on a 60^3 grid with diagonal shift
1e-3 (n = 216,000), FP64, MMD ordering, right-hand sides standard-normal from
seed 0 with nrhs in {1, 16}.  Synthetic data of that shape; the factor arena
(1.4 GB) is far larger than L2, so no flush is needed between steps.

One step = DistributeMatrix (values already in HBM) + Factorize + Solve(nrhs=1)
+ Solve(nrhs=16).  `value` is factor TFLOP/s using the reference's own flop
statistic (sum of squared column counts); solves/s, backward errors, p50/p99
step latency, a roofline of the dominant kernel, the end-to-end number through
the host-buffer API and the CPU baseline ride on the same JSON line.

Multi-GPU: one factorization does not shard, so N ranks run N independent
replicas (weak scaling); timings are the max over ranks.

--impl reference times the CPU restatement of the reference's numeric path
(oracle/, OpenBLAS on all host cores) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes (read + write) of one k_factor_persistent launch on the 60^3 workload, from ncu
# (dram__bytes.sum.per_second x gpu__time_duration; profiles/factor_persistent_lap3d60_ncu.md)
FACTOR_TRAFFIC_BYTES = 15.57e9
METRIC = "factor TFLOP/s (FP64 supernodal Cholesky, flops = sum of squared column counts)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--grid", type=int, default=60, help="grid edge of the 3D Laplacian (60 = the named workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-precision", action="store_true", help="skip the FP64 vs FP32+IR comparison")
    ap.add_argument("--precision-grid", type=int, default=80,
                    help="grid edge of the 27-point stencil of the precision comparison (80 = the named workload)")
    ap.add_argument("--batch-systems", type=int, default=2000,
                    help="systems of the batching workload (2000 = the named workload; the host analysis of its "
                         "random graphs takes about two minutes)")
    ap.add_argument("--serve-requests", type=int, default=10000,
                    help="requests of the serving workload (10000 = the named workload), run whole by the "
                         "continuous-batching loop at capacity")
    ap.add_argument("--serve-sample", type=int, default=1000,
                    help="requests of the stream's start run back to back (FP64 baseline) and with Poisson "
                         "arrivals at 0.7x capacity (a rate: it does not depend on how many follow)")
    ap.add_argument("--serve-fp64-batching", action="store_true",
                    help="also run the continuous-batching loop in FP64 at capacity")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-ldl", action="store_true", help="skip the LDL^T vs Cholesky comparison")
    ap.add_argument("--no-serve", action="store_true")
    return ap.parse_args()


def build_matrix(k):
    from sympack_b200 import generators as G
    return G.laplacian_3d(k, k, k, shift=1e-3)


def backward_error(A, x, b):
    """||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf), per right-hand side (max), in FP64."""
    import scipy.sparse as sp
    n = A.size
    L = sp.csc_matrix((A.nzvalLocal, A.rowind - 1, A.colptr - 1), shape=(n, n))
    full = L + sp.tril(L, -1).T
    r = b.reshape(n, -1) - full @ x.reshape(n, -1)
    anorm = abs(full).sum(axis=1).max()
    r2, x2, b2 = r, x.reshape(n, -1), b.reshape(n, -1)
    eta = np.abs(r2).max(0) / (anorm * np.abs(x2).max(0) + np.abs(b2).max(0))
    return float(eta.max())


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_fp64_peak(torch, dev):
    """cuBLAS DGEMM throughput on this GPU (TFLOP/s): the FP64 tensor-pipe denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(3):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "MEASURED_PEAKS.json"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def cpu_baseline_run(n, cp, ri, v, sym, flops, steps=1, warmup=0):
    """CPU restatement of the reference numeric path (oracle, OpenBLAS, all host cores).
    Per step: DistributeMatrix + Factorize + Solve(nrhs 1) + Solve(nrhs 16), each timed."""
    from oracle import numeric
    cores = os.cpu_count() or 1
    f = numeric.OracleFactor(n, sym, threads=cores)
    rng = np.random.default_rng(0)
    b1 = rng.standard_normal((n, 1))
    b16 = rng.standard_normal((n, 16))
    dist, fac, s1, s16 = [], [], [], []
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        f.distribute(cp, ri, v)
        t1 = time.perf_counter()
        f.factorize()
        t2 = time.perf_counter()
        f.solve(b1)
        t3 = time.perf_counter()
        f.solve(b16)
        t4 = time.perf_counter()
        if it >= warmup:
            dist.append(t1 - t0)
            fac.append(t2 - t1)
            s1.append(t3 - t2)
            s16.append(t4 - t3)
    mean = lambda a: sum(a) / len(a)
    return dict(tflops=flops / mean(fac) / 1e12, factor_s=mean(fac), distribute_s=mean(dist),
                solve1_s=mean(s1), solve16_s=mean(s16), cores=cores,
                # the GPU arm's e2e work: DistributeMatrix + Factorize + Solve(16) + GetSolution
                e2e_tflops=flops / (mean(dist) + mean(fac) + mean(s16)) / 1e12,
                step_s=[a + b + c + d for a, b, c, d in zip(dist, fac, s1, s16)])


def oracle_symbolic(n, cp, ri):
    """The workload's symbolic analysis from the oracle alone (the reference's own
    compiled MMD plus the Python restatement of the rest of the chain); loads no
    product library."""
    from oracle import symbolic_oracle
    return symbolic_oracle.reference_symbolic(n, cp, ri)


def bench_config(n, nnz_l, flops, gpus):
    """`config` of the JSON line; both arms emit exactly this dict."""
    k = round(n ** (1.0 / 3.0))
    workload = f"3D 7-point Laplacian {k}^3 + 1e-3 I (n={n}), FP64, MMD, nrhs 1 and 16"
    return {"workload": workload, "n": n, "nnz_L": int(nnz_l), "flops_stat": float(flops), "nrhs": [1, 16],
            "parallelism": f"replicas x{gpus}" if gpus > 1 else "1 GPU",
            "l2": "no flush: every step reads and writes the whole factor (1.4 GB), far above the 126 MB L2"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n, cp, ri, v = build_matrix(args.grid)
    sym, flops, nnz_l = oracle_symbolic(n, cp, ri)
    r = cpu_baseline_run(n, cp, ri, v, sym, flops, steps=args.steps, warmup=args.warmup)
    st = r["step_s"]
    line = {
        "impl": "reference", "metric": METRIC, "value": r["tflops"], "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(st) / len(st),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(n, nnz_l, flops, args.gpus),
        "factor_ms": 1e3 * r["factor_s"],
        "solves_per_s": {"nrhs1": 1.0 / r["solve1_s"], "nrhs16": 16.0 / r["solve16_s"]},
        "solve_ms": {"nrhs1": 1e3 * r["solve1_s"], "nrhs16": 1e3 * r["solve16_s"]},
        "cpu_baseline": {"value": r["tflops"], "unit": "TFLOP/s", "cores": r["cores"], "kind": "port",
                         "sample": "per step the full workload: DistributeMatrix + Factorize + Solve(nrhs 1) + "
                                   "Solve(nrhs 16); CPU restatement of the reference 2D cell algorithm "
                                   "(oracle/numeric_oracle.c over OpenBLAS); symbolic analysis from the "
                                   "reference's compiled MMD + the Python restatement of the chain"},
        "e2e": {"value": r["e2e_tflops"], "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "ms_per_step": 1e3 * (r["distribute_s"] + r["factor_s"] + r["solve16_s"]),
                "note": "flops_stat / (DistributeMatrix + Factorize + Solve(16 RHS)), the GPU arm's e2e work"},
    }
    print(json.dumps(line), flush=True)
    return 0


def precision_comparison(torch, dev, stream, grid=80, reps=2):
    """Time-to-solution (DistributeMatrix + Factorize + Solve(nrhs=1)) of the plain FP64
    path and of the FP32 factor + FP64 refinement on the 27-point stencil, for the two
    diagonal shifts of the precision workload.  Same matrices, same ordering."""
    from sympack_b200 import DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions
    n, cp, ri, v = G.stencil27(grid, grid, grid, 1e-2, seed=0)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    T = symPACKMatrix2D()
    T.Init(symPACKOptions(device=-1))
    T.SymbolicFactorization(A)
    flops = T.info().flops_stat
    b = torch.from_numpy(np.random.default_rng(0).standard_normal(n)).to(dev)
    x = torch.empty_like(b)
    out = {"workload": f"3D 27-point stencil {grid}^3 (n={n}), off-diagonals U[-1,0), seed 0, nrhs 1",
           "flops_stat": flops}
    # plan of each precision: the fastest factorization schedule (one persistent launch, or
    # the level-ordered launch sequence) and outer block (256 or 512 columns) on this matrix,
    # timed once, outside the comparison
    _, _, _, v0 = G.stencil27(grid, grid, grid, 1e-2, seed=0)
    dv0 = torch.from_numpy(v0).to(dev)
    handles, plans = {}, {}
    for prec in ("FP64", "FP32_IR"):
        best = None
        for sched in ("persistent", "steps"):
            M = symPACKMatrix2D()
            M.Init(symPACKOptions(device=dev.index, precision=prec, factor_schedule=sched))
            M.SymbolicFactorizationFrom(T)
            M.SetStream(stream.cuda_stream)
            mine = None
            for onb in (256, 512):
                M.Replan(0, 0, onb)
                ts = []
                for r in range(3):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    M.DistributeMatrixDevice(dv0.data_ptr())
                    M.Factorize()
                    e1.record(stream)
                    torch.cuda.synchronize()
                    if r:
                        ts.append(e0.elapsed_time(e1))
                plans.setdefault(prec, {})[f"{sched},{onb}"] = round(min(ts), 2)
                if mine is None or min(ts) < mine[1]:
                    mine = (onb, min(ts))
            if best is None or mine[1] < best[2]:
                if best is not None:
                    best[3].close()
                M.Replan(0, 0, mine[0])
                best = (sched, mine[0], mine[1], M)
            else:
                M.close()
        handles[prec] = best[3]
        plans[prec]["chosen"] = {"factor_schedule": best[0], "outer_nb": best[1], "factor_ms": best[2]}
    T.close()
    out["plans_factor_ms"] = plans
    for delta in (1e-2, 1e-5):
        _, _, _, vd = G.stencil27(grid, grid, grid, delta, seed=0)
        dv = torch.from_numpy(vd).to(dev)
        res = {}
        for prec, M in handles.items():
            times = []
            for r in range(reps + 1):
                e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
                e0.record(stream)
                M.DistributeMatrixDevice(dv.data_ptr())
                M.Factorize()
                e1.record(stream)
                M.SolveDevice(b.data_ptr(), x.data_ptr(), 1, n)
                e2.record(stream)
                torch.cuda.synchronize()
                if r:
                    times.append((e0.elapsed_time(e1), e1.elapsed_time(e2)))
            fac = min(t[0] for t in times)
            sol = min(t[1] for t in times)
            inf = M.info()
            Ad = DistSparseMatrix.from_lower_csc(n, cp, ri, vd)
            eta = backward_error(Ad, x.cpu().numpy(), b.cpu().numpy())
            res[prec] = {"factor_ms": fac, "solve_ms": sol, "time_to_solution_ms": fac + sol,
                         "factor_tflops": flops / (fac * 1e-3) / 1e12, "backward_error": eta,
                         "ir_iterations": inf.ir_iterations if prec == "FP32_IR" else 0}
        res["speedup_time_to_solution"] = res["FP64"]["time_to_solution_ms"] / res["FP32_IR"]["time_to_solution_ms"]
        out[f"delta={delta:g}"] = res
        if delta == 1e-2:  # kernel breakdown of one eager (profiled) factor + solve per precision
            for prec, M in handles.items():
                M.SetProfiling(True)
                M.DistributeMatrixDevice(dv.data_ptr())
                M.Factorize()
                M.SolveDevice(b.data_ptr(), x.data_ptr(), 1, n)
                prof = M.GetProfile()
                M.SetProfiling(False)
                out.setdefault("kernels_profiled", {})[prec] = {
                    k: {"ms": round(p["ms"], 3), "launches": p["launches"],
                        "tflops": round(p["flops"] / (p["ms"] * 1e-3) / 1e12, 2) if p["ms"] > 0 else 0.0}
                    for k, p in prof.items() if p["launches"]}
    for M in handles.values():
        M.close()
    torch.cuda.empty_cache()
    return out


def ldl_comparison(torch, dev, stream, grid=60, qd_grid=50, reps=2):
    """LDL^T (the reference's -fact LDL) next to Cholesky on the headline matrix (same
    analysis, same flop statistic), and LDL^T alone on a quasi-definite indefinite
    matrix of the same kind of grid, which Cholesky rejects.  Device-resident values,
    factor and nrhs-1 solve timed with CUDA events (best of reps)."""
    from sympack_b200 import DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions

    def run(n, cp, ri, v, dec):
        A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
        M = symPACKMatrix2D()
        M.Init(symPACKOptions(device=dev.index, decomposition=dec))
        M.SymbolicFactorization(A)
        M.SetStream(stream.cuda_stream)
        dv = torch.from_numpy(v).to(dev)
        b = torch.from_numpy(np.random.default_rng(0).standard_normal(n)).to(dev)
        x = torch.empty_like(b)
        fac, sol = [], []
        for r in range(reps + 1):
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            M.DistributeMatrixDevice(dv.data_ptr())
            M.Factorize()
            e1.record(stream)
            M.SolveDevice(b.data_ptr(), x.data_ptr(), 1, n)
            e2.record(stream)
            torch.cuda.synchronize()
            if r:
                fac.append(e0.elapsed_time(e1))
                sol.append(e1.elapsed_time(e2))
        flops = M.info().flops_stat
        out = {"factor_ms": min(fac), "solve_ms": min(sol), "factor_tflops": flops / (min(fac) * 1e-3) / 1e12,
               "backward_error": backward_error(A, x.cpu().numpy(), b.cpu().numpy())}
        M.close()
        torch.cuda.empty_cache()
        return out

    n, cp, ri, v = build_matrix(grid)
    res = {"workload": f"3D 7-point Laplacian {grid}^3 + 1e-3 I (n={n}), MMD, nrhs 1",
           "LL": run(n, cp, ri, v, "LL"), "LDL": run(n, cp, ri, v, "LDL")}
    res["ldl_over_ll_factor_time"] = res["LDL"]["factor_ms"] / res["LL"]["factor_ms"]
    qn, qcp, qri, qv = G.quasi_definite_3d(qd_grid, qd_grid, qd_grid, 0.3, 1e-2, seed=0)
    res["indefinite"] = {"workload": f"quasi-definite 27-point {qd_grid}^3 (n={qn}), 30% negative vertices, "
                                     f"delta 1e-2, seed 0, MMD, nrhs 1",
                         "LDL": run(qn, qcp, qri, qv, "LDL")}
    return res


def per_system_backward_error(systems, offs, x, b):
    from sympack_b200 import DistSparseMatrix
    eta = 0.0
    for k, s in enumerate(systems):
        lo, hi = int(offs[k]), int(offs[k + 1])
        eta = max(eta, backward_error(DistSparseMatrix.from_lower_csc(*s), x[lo:hi], b[lo:hi]))
    return eta


def batching_comparison(torch, dev, stream, count, seed=0, subset=64, tune_systems=200):
    """Batching form: `count` uneven systems factored together (FP64: every task of every
    system in one persistent launch; FP32 + refinement: each etree level of every system in
    the same launches), in FP64 and FP32 + refinement, with tile shapes picked by the
    autotuner on the first `tune_systems` systems (each candidate re-plans the batch, so the
    candidates are timed on that sample and the winner plans the whole batch); beside it the
    first `subset` systems factored one by one versus as one batch."""
    from sympack_b200 import (DistSparseMatrix, SymPACKError, autotune, generators as G, symPACKMatrix2D,
                              symPACKOptions)
    SPB_ERR_OOM = -3  # include/sympack_b200.h
    systems = G.batch_systems(count, 500, 20000, seed=seed)
    n, cp, ri, v, offs = G.block_diagonal(systems)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    b = np.random.default_rng(seed).standard_normal((n, 1))
    db = torch.from_numpy(b).to(dev)
    dx = torch.empty_like(db)
    out = {"workload": f"{count} SPD systems, n log-uniform [500, 20000]; even: 2D/3D Laplacians on random grids, "
                       f"odd: random graphs avg degree 10, off-diagonals U[-1,0), dominance 1.05 (seed {seed})",
           "systems": count, "n_total": n}
    T = symPACKMatrix2D()
    T.Init(symPACKOptions(device=-1, factor_schedule="steps"))  # analysis only: no task graph
    t0 = time.perf_counter()
    T.SymbolicFactorizationBatch(A, offs)
    out["symbolic_s"] = time.perf_counter() - t0
    inf = T.info()
    flops = inf.flops_stat
    out.update(flops_stat=flops, nnz_L=inf.nnz_l, nsuper=inf.nsuper, etree_levels=inf.nlevels,
               max_width=inf.max_width)
    sample = systems[:min(tune_systems, count)]
    tn, tcp, tri, tv, toffs = G.block_diagonal(sample)
    At = DistSparseMatrix.from_lower_csc(tn, tcp, tri, tv)
    for prec in ("FP64", "FP32_IR"):
        S = symPACKMatrix2D()
        S.Init(symPACKOptions(device=dev.index, precision=prec))
        S.SymbolicFactorizationBatch(At, toffs)
        tune = autotune.tune(S, At, toffs, reps=1, use_cache=False)
        S.close()
        # the FP32 tiles read TMA-fed split copies of the panels when they fit the device
        # (they double the FP32 arena), else stage and split their operands per tile
        engines = [{}] if prec == "FP64" else [{"fp32_engine": "tcgen05-tma"}, {"fp32_engine": "tcgen05"}]
        for eng in engines:
            M = symPACKMatrix2D()
            M.Init(symPACKOptions(device=dev.index, precision=prec, plan_small_max_w=tune["small_max_w"],
                                  plan_big_tile_rows=tune["big_tile_rows"], plan_outer_nb=tune["outer_nb"], **eng))
            try:
                M.SymbolicFactorizationFrom(T)
                break
            except SymPACKError as e:
                M.close()
                torch.cuda.empty_cache()
                if e.code != SPB_ERR_OOM or eng is engines[-1]:
                    raise
        M.SetStream(stream.cuda_stream)
        times = []
        for r in range(3):
            M.DistributeMatrix(A)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            M.Factorize()
            e1.record(stream)
            M.SolveDevice(db.data_ptr(), dx.data_ptr(), 1, n)
            e2.record(stream)
            torch.cuda.synchronize()
            if r:
                times.append((e0.elapsed_time(e1), e1.elapsed_time(e2)))
        fac = min(t[0] for t in times)
        sol = min(t[1] for t in times)
        mi = M.info()
        out[prec] = {"factor_ms": fac, "solve_ms": sol, "factor_tflops": flops / (fac * 1e-3) / 1e12,
                     "systems_per_s": count / ((fac + sol) * 1e-3),
                     "backward_error_max_over_systems": per_system_backward_error(systems, offs, dx.cpu().numpy(), b),
                     "ir_iterations": mi.ir_iterations if prec == "FP32_IR" else 0,
                     "factor_launches": mi.factor_launches, "device_bytes": mi.device_bytes,
                     "fp32_engine": eng.get("fp32_engine"),
                     "autotuned_plan": {"small_max_w": tune["small_max_w"], "big_tile_rows": tune["big_tile_rows"],
                                        "outer_nb": tune["outer_nb"], "tuned_on_systems": len(sample),
                                        "candidates_ms": {k: round(v * 1e3, 3) for k, v in tune["times"].items()}}}
        M.close()
    T.close()
    # one by one versus batched, on the first `subset` systems (FP64, default plan)
    sub = systems[:subset]
    sn, scp, sri, sv, soffs = G.block_diagonal(sub)
    seq_ms = 0.0
    for s in sub:
        As = DistSparseMatrix.from_lower_csc(*s)
        M = symPACKMatrix2D()
        M.Init(symPACKOptions(device=dev.index))
        M.SymbolicFactorization(As)
        M.SetStream(stream.cuda_stream)
        M.DistributeMatrix(As)
        M.Factorize()  # graph capture outside the timing
        M.DistributeMatrix(As)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        M.Factorize()
        e1.record(stream)
        torch.cuda.synchronize()
        seq_ms += e0.elapsed_time(e1)
        M.close()
    As = DistSparseMatrix.from_lower_csc(sn, scp, sri, sv)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=dev.index))
    M.SymbolicFactorizationBatch(As, soffs)
    M.SetStream(stream.cuda_stream)
    M.DistributeMatrix(As)
    M.Factorize()
    M.DistributeMatrix(As)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    M.Factorize()
    e1.record(stream)
    torch.cuda.synchronize()
    out["one_by_one_vs_batched"] = {"systems": subset, "one_by_one_factor_ms": seq_ms,
                                    "batched_factor_ms": e0.elapsed_time(e1),
                                    "speedup": seq_ms / e0.elapsed_time(e1)}
    M.close()
    torch.cuda.empty_cache()
    return out


def serving_comparison(torch, dev, count, seed=0, load=0.7, sample=1000, fp64_batching=False, check_every=25):
    """Serving form on the request stream: (1) back-to-back plain FP64, one request after
    the other, on the stream's first `sample` requests (a sequential baseline: its rate
    does not depend on how many requests follow); (2) the continuous-batching loop (8 slots,
    right-hand sides merged per factor) in FP32 + refinement with all `count` requests
    submitted at once, which gives its capacity (and, with `fp64_batching`, the same loop in
    FP64); (3) the FP32 + refinement loop on the first `sample` requests with Poisson
    arrivals at `load` x its capacity, which gives p50 / p99 latency at a sustainable rate.
    Every `check_every`-th result is checked on the host: its backward error
    ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) (FP64 results do not compute it on
    the device)."""
    from sympack_b200 import serving as S
    mk = lambda k: S.request_stream(k, 1.0, seed=seed)
    patterns = {}
    for _, r in mk(count):
        if r.spec[0] is not None:
            patterns[(r.spec[0].kind, r.spec[0].k)] = r.spec[0]

    def preload(svc):  # symbolic analyses of the stream's patterns, outside the timed region
        from sympack_b200 import DistSparseMatrix
        for P in patterns.values():
            svc._ensure_pattern(DistSparseMatrix.from_lower_csc(P.n, P.colptr, P.rowind, P.base))
        for f in list(svc._patterns.values()):
            f.result()

    def run(precision, slots, merge, rate, k):
        stream = [(t / rate if rate else 0.0, r) for t, r in mk(k)]
        for i, (_, r) in enumerate(stream):
            r.keep = i % check_every == 0
        specs = {r.factor_id: (r.spec[0], r.spec[1]) for _, r in stream if r.kind == "factor_solve"}
        svc = S.SolverService(device=dev.index, precision=precision, max_inflight=slots, max_batch_rhs=merge)
        preload(svc)
        if rate is None:  # back to back: each request starts when the previous one ends
            t0 = time.perf_counter()
            for _, r in stream:
                svc.submit(S.materialise(r)).result()
            wall = time.perf_counter() - t0
        else:
            wall = S.replay(svc, stream, timeout=3600)
        res = [r.future.result() for _, r in stream]
        svc.close()
        torch.cuda.empty_cache()
        # host check of the kept results, against the matrix of the request's factor (drawn
        # again from its pattern and seed)
        eta = 0.0
        for (_, r), x in zip(stream, res):
            if x.x is not None:
                P, sd = specs[r.factor_id]
                eta = max(eta, backward_error(P.matrix(sd), x.x, r.rhs))
        out = {"requests": k, "solves_per_s": k / wall, "wall_s": wall, **S.latency_summary([r for _, r in stream]),
               "service_p50_ms": float(np.percentile([(r.t_done - r.t_start) * 1e3 for _, r in stream], 50)),
               "service_p99_ms": float(np.percentile([(r.t_done - r.t_start) * 1e3 for _, r in stream], 99)),
               "max_backward_error_device": max((x.backward_error for x in res if x.backward_error >= 0), default=None),
               "max_backward_error_host_checked": eta, "host_checked_results": sum(1 for x in res if x.x is not None)}
        out.update({kk: int(v) for kk, v in svc.stats.items()})
        return out

    sample = min(sample, count)
    base = run("FP64", 1, 1, None, sample)
    cap = run("FP32_IR", 8, 64, 0.0, count)
    rate = load * cap["solves_per_s"]
    lat = run("FP32_IR", 8, 64, rate, sample)
    lat["arrival_rate_per_s"] = rate
    out = {
        "workload": f"{count} requests, Poisson arrivals, 30% factor+solve on fresh 27-point stencil (delta 1e-2) "
                    f"or 2D Laplacian matrices, n 1k-216k on a grid ladder, 70% solve-only against the 8 latest "
                    f"factors, nrhs U{{1..64}} (seed {seed})",
        "requests": count,
        "back_to_back_fp64": base,
        "continuous_batching_fp32_ir_capacity": cap,
        "continuous_batching_fp32_ir_at_load": lat,
        "speedup_solves_per_s_at_load": lat["solves_per_s"] / base["solves_per_s"],
        "speedup_capacity": cap["solves_per_s"] / base["solves_per_s"],
    }
    if fp64_batching:
        cap64 = run("FP64", 8, 64, 0.0, count)
        out["continuous_batching_fp64_capacity"] = cap64
        out["speedup_capacity_batching_fp64"] = cap64["solves_per_s"] / base["solves_per_s"]
        out["speedup_capacity_precision_fp32_ir_over_fp64"] = cap["solves_per_s"] / cap64["solves_per_s"]
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    from sympack_b200 import DistSparseMatrix, symPACKMatrix2D, symPACKOptions

    from sympack_b200 import replicas
    world, rank, local = replicas.world_info()
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    n, cp, ri, v = build_matrix(args.grid)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=local))
    t0 = time.perf_counter()
    M.SymbolicFactorization(A)
    symb_s = time.perf_counter() - t0
    info = M.info()
    flops = info.flops_stat
    stream = torch.cuda.current_stream(dev)
    M.SetStream(stream.cuda_stream)

    rng = np.random.default_rng(0)
    b1 = rng.standard_normal((n, 1))
    b16 = np.asfortranarray(rng.standard_normal((n, 16)))
    d_vals = torch.from_numpy(A.nzvalLocal).to(dev)
    d_b1 = torch.from_numpy(b1).to(dev)
    d_b16 = torch.from_numpy(np.ascontiguousarray(b16.T)).to(dev)  # column-major n x 16
    d_x1 = torch.empty_like(d_b1)
    d_x16 = torch.empty_like(d_b16)

    def step():
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        ev[0].record(stream)
        M.DistributeMatrixDevice(d_vals.data_ptr())
        ev[4].record(stream)  # the factorization launch alone: ev[4] -> ev[1]
        M.Factorize()
        ev[1].record(stream)
        M.SolveDevice(d_b1.data_ptr(), d_x1.data_ptr(), 1, n)
        ev[2].record(stream)
        M.SolveDevice(d_b16.data_ptr(), d_x16.data_ptr(), 16, n)
        ev[3].record(stream)
        return ev

    def barrier():
        replicas.barrier(dist, torch.cuda.synchronize)

    for _ in range(args.warmup):
        step()
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    evs = [step() for _ in range(args.steps)]
    barrier()
    clocks = sampler.stop()
    fac = [e[0].elapsed_time(e[1]) for e in evs]
    fac_kernel = [e[4].elapsed_time(e[1]) for e in evs]  # counter reset + the persistent factorization
    s1 = [e[1].elapsed_time(e[2]) for e in evs]
    s16 = [e[2].elapsed_time(e[3]) for e in evs]
    tot = [e[0].elapsed_time(e[3]) for e in evs]
    fac_ms, s1_ms, s16_ms, tot_ms = replicas.max_over_ranks([sum(fac), sum(s1), sum(s16), sum(tot)], dev, dist)

    x1 = d_x1.cpu().numpy()
    x16 = np.asfortranarray(d_x16.cpu().numpy().T)
    bwd1 = backward_error(A, x1, b1)
    bwd16 = backward_error(A, x16, b16)

    # end to end through the host-buffer API (pinned host values / RHS, solution read back)
    h_vals = torch.from_numpy(A.nzvalLocal).pin_memory()
    h_b16 = torch.from_numpy(np.ascontiguousarray(b16.T)).pin_memory()
    h_out = torch.empty_like(h_b16).pin_memory()
    from sympack_b200 import _native as Nn
    import ctypes as C
    lib = Nn.load()
    dp = lambda t: C.cast(C.c_void_p(t.data_ptr()), Nn._DP)

    def e2e_step():
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for rc in (lib.spb_distribute(M._h, dp(h_vals)), lib.spb_factorize(M._h),
                   lib.spb_solve(M._h, dp(h_b16), 16, n), lib.spb_get_solution(M._h, dp(h_out), 16, n)):
            if rc != 0:
                raise RuntimeError(f"e2e call failed ({rc}): {lib.spb_last_error(M._h).decode()}")
        e.record(stream)
        return s, e

    for _ in range(max(1, args.warmup)):
        e2e_step()
    barrier()
    e2e_ev = [e2e_step() for _ in range(args.steps)]
    barrier()
    e2e_ms = replicas.max_over_ranks([sum(s.elapsed_time(e) for s, e in e2e_ev)], dev, dist)[0]
    bwd_e2e = backward_error(A, np.asfortranarray(h_out.numpy().T), b16)

    # the dominant kernel: the persistent FP64 factorization (every task of the factorization
    # in one launch), timed by the events around it in the timed steps above
    peaks, peak_src = measured_peaks()
    fp64_peak = measured_fp64_peak(torch, dev)
    fk_ms = sum(fac_kernel) / len(fac_kernel)
    roofline = {"kernel": "k_factor_persistent", "bound": "tensor",
                "achieved": flops / (fk_ms * 1e-3) / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": None, "launch_ms": fk_ms,
                # dram__bytes (read + write) of one launch on this workload, from the ncu capture
                # summarised in profiles/factor_persistent_lap3d60_ncu.md
                "traffic": FACTOR_TRAFFIC_BYTES if args.grid == 60 else None,
                "algorithmic_bytes": 2.0 * info.arena_bytes,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (no FP64 figure in " + peak_src + ")"}
    roofline["frac"] = roofline["achieved"] / roofline["peak"]
    # where the factorization's CTA time goes: one traced factorization (outside the timing)
    M.SetFactorTrace(True)
    M.DistributeMatrixDevice(d_vals.data_ptr())
    M.Factorize()
    tr, tkinds = M.GetFactorTrace()
    M.SetFactorTrace(False)
    tr = tr.astype(np.int64)
    busy = (tr[:, 2] - tr[:, 1]).astype(np.float64)
    span = float(tr[:, 2].max() - tr[:, 0].min())
    nsm = len(np.unique(tr[:, 3]))
    names = ["small_panel", "diagonal_block", "trsm_tile", "tile_64x64_fma", "tile_128x64_dmma"]
    roofline["task_breakdown"] = {
        names[k]: {"tasks": int(np.sum(tkinds == k)), "cta_ms": float(busy[tkinds == k].sum() / 1e6),
                   "share_of_busy": float(busy[tkinds == k].sum() / busy.sum())} for k in range(5)}
    # CTAs running a task, averaged over the launch and the SMs (two CTAs fit on an SM)
    roofline["mean_busy_ctas_per_sm"] = float(busy.sum() / (span * nsm))
    # one profiled step (eager launches of the level-ordered sequence, per-launch CUDA events):
    # the solve sweeps' byte count and the per-kind times of the step schedule
    M.SetProfiling(True)
    M.DistributeMatrixDevice(d_vals.data_ptr())
    M.Factorize()
    M.SolveDevice(d_b16.data_ptr(), d_x16.data_ptr(), 16, n)
    prof = M.GetProfile()
    M.SetProfiling(False)
    sf, sb = prof["solve_forward"], prof["solve_backward"]
    roofline_solve = {"kernel": "solve_forward+solve_backward", "bound": "hbm", "unit": "GB/s",
                      "achieved": (sf["bytes"] + sb["bytes"]) / ((sf["ms"] + sb["ms"]) * 1e-3) / 1e9,
                      "peak": peaks.get("hbm_gbs"), "peak_source": peak_src, "nrhs": 16}
    roofline_solve["frac"] = roofline_solve["achieved"] / roofline_solve["peak"]
    kernels = {k: {"ms": round(p["ms"], 4), "launches": p["launches"]} for k, p in prof.items() if p["launches"]}

    # the precision, LDL^T, batching and serving comparisons are one-GPU measurements: with
    # several replicas only the headline line is measured
    # a failing comparison is reported in its own key; the headline line still prints
    def section(enabled, fn, *a, **kw):
        if not enabled or world != 1:
            return None
        try:
            return fn(*a, **kw)
        except Exception as e:  # noqa: BLE001
            print(f"bench: {fn.__name__} failed: {e!r}", file=sys.stderr, flush=True)
            return {"error": repr(e)[:400]}

    precision = section(not args.no_precision, precision_comparison, torch, dev, stream, grid=args.precision_grid)
    # roofline of the FP32 update tiles: 3xTF32 issues three MMAs per useful product; tcgen05
    # runs kind::tf32 at half the dense kind::f16 rate, so the TF32 peak is half the measured bf16
    try:
        tiles = precision["kernels_profiled"]["FP32_IR"]["gemm_dmma"]
        tf32_peak = peaks["bf16_tflops"] / 2
        precision["fp32_tile_roofline"] = {
            "kernel": "k_gemm_tc32w", "bound": "tensor", "unit": "TFLOP/s",
            "useful": tiles["tflops"], "mma_work": 3 * tiles["tflops"], "peak": tf32_peak,
            "frac": 3 * tiles["tflops"] / tf32_peak,
            "peak_source": "half the dense bf16 rate of " + peak_src + " (tcgen05 kind::tf32 runs at half kind::f16)"}
    except (KeyError, TypeError):
        pass
    ldl = section(not args.no_ldl, ldl_comparison, torch, dev, stream, grid=args.grid)
    batching = section(not args.no_batch, batching_comparison, torch, dev, stream, args.batch_systems)
    serving = section(not args.no_serve, serving_comparison, torch, dev, args.serve_requests,
                      sample=args.serve_sample, fp64_batching=args.serve_fp64_batching)

    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        sym, _, _ = oracle_symbolic(n, cp, ri)
        r = cpu_baseline_run(n, cp, ri, v, sym, flops, steps=1, warmup=0)
        cpu = {"value": r["tflops"], "unit": "TFLOP/s", "cores": r["cores"], "kind": "port",
               "sample": "one full step of the workload (DistributeMatrix + Factorize + Solve(nrhs 1) + "
                         "Solve(nrhs 16), timed separately); CPU restatement of the reference 2D cell algorithm "
                         "over OpenBLAS",
               "factor_s": r["factor_s"], "solve1_s": r["solve1_s"], "solve16_s": r["solve16_s"],
               "e2e_value": r["e2e_tflops"]}

    K = args.steps
    # per step: assemble, the factorization (one persistent launch), then two solves (permute in,
    # forward, backward, permute out), the first one after the factorization also computing the
    # diagonal super-block inverses
    launches_per_step = 1 + info.factor_launches + 4 + 4 + (1 if info.inverse_bytes else 0)
    if rank == 0:
        line = {
            "metric": METRIC, "value": replicas.job_rate(flops * K, world, fac_ms) / 1e12, "unit": "TFLOP/s",
            "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": tot_ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(n, info.nnz_l, flops, world),
            "analysis": {"flops_exec": info.flops_exec, "nsuper": info.nsuper, "etree_levels": info.nlevels,
                         "factor_arena_gb": info.arena_bytes / 1e9, "symbolic_s": symb_s},
            "factor_ms": fac_ms / K,
            "factor_schedule": "persistent (one launch per factorization)" if info.factor_launches == 1 else "steps",
            "solves_per_s": {"nrhs1": world * K / (s1_ms * 1e-3), "nrhs16": world * 16 * K / (s16_ms * 1e-3)},
            "solve_ms": {"nrhs1": s1_ms / K, "nrhs16": s16_ms / K},
            "backward_error": {"nrhs1": bwd1, "nrhs16": bwd16, "e2e_nrhs16": bwd_e2e},
            "latency_ms": {"p50": float(np.percentile(tot, 50)), "p99": float(np.percentile(tot, 99))},
            "roofline": roofline, "roofline_solve": roofline_solve, "kernels_profiled_step": kernels,
            "precision_form": precision,
            "ldl_form": ldl,
            "batching_form": batching,
            "serving_form": serving,
            "cpu_baseline": cpu,
            "e2e": {"value": world * flops * K / (e2e_ms * 1e-3) / 1e12, "unit": "TFLOP/s",
                    "h2d_bytes_per_step": int(A.nnz * 8 + n * 16 * 8), "d2h_bytes_per_step": int(n * 16 * 8),
                    "ms_per_step": e2e_ms / K,
                    "note": "DistributeMatrix from pinned host values + Factorize + Solve(16 host RHS) + GetSolution"},
            "clocks": clocks,
            "gpu_launches": launches_per_step * K,
        }
        print(json.dumps(line), flush=True)
    M.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
