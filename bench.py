#!/usr/bin/env python
"""Benchmark of the pattern-evaluator fitting path on B200.

Workload (one step): the 20M-row, 8-pattern fit — 20,000,000 random-play
positions with empty counts uniform in 20..40, patterns edge+2X, 3x3 corner,
2x5 corner, main diagonal, rows 2/3/4 and the 7-square diagonal, each under
the 8 board symmetries (expanded layout: 166,212 columns, 64 entries per
row, 1.28e9 entries), seeded synthetic targets.  A step is FitWeights on
device-resident positions and targets: indexing, CSR and transposed-copy
build, Jacobi, and mixed-precision Jacobi-PCG to a relative normal-equation
residual of 1e-8.  The metric is the time of that step (lower is better).

Beside it on the same line: the plain FP64 GPU path (the fit on the rows
layout, and FP64 and mixed solves on one blocked CSR, which isolates the
precision); LSQR solves of the same system (``--lsqr``); the reference's
own code on the host cores solving the same system (the CPU baseline, one
full step) and the check of every device solution against it (FP64
normal-equation residual with the reference's products, largest weight
difference on the columns with entries); short runs of the batched and
evaluator workloads (``--no-summaries`` leaves them out).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Other workloads: ``--workload batched`` — the 60 per-empty-count fits
(16.6M rows in total) as one batched mixed solve; ``--workload evaluator`` —
one training epoch of the differentiable evaluator (8M positions, Adam on
Huber + L2 over 65,536-row minibatches, each minibatch step one CUDA graph).
``--impl reference`` times the reference's own CPU code on the selected
workload; for the single fit every step is the whole 20M-row workload, with
inputs from the oracle's restatement of the seeded generator.

N > 1 runs under torchrun, one rank per GPU: the single workload becomes one
fit sharded by rows (each rank holds a block range of the 20M rows; one
all-reduce per PCG iteration; strong scaling), the batched and evaluator
workloads run one independently seeded replica per rank (their fits are
independent; no collective on the data path).  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "time to rel. residual 1e-8: mixed/batched vs plain FP64 GPU; SpMV HBM GB/s"
PATTERNS_8 = [0x42FF, 0x070707, 0x1F1F, 0x8040201008040201, 0xFF00, 0xFF0000, 0xFF000000, 0x0080402010080402]
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes (read + write) per entry of the blocked FP32 products, measured
# with ncu (dram__bytes_read.sum + dram__bytes_write.sum of one launch) on a
# 2M-row launch of the same kernels, 128M entries; traffic grows with the
# entries, so a full launch's traffic is this times its entries.
NCU_DRAM_BYTES_PER_ENTRY = {"aty_f32": (563.91e6 + 33.30e6) / 128e6, "ax_f32": (288.12e6 + 4.19e6) / 128e6}


def ncu_traffic(kernel: str, entries: int):
    for suffix, per in NCU_DRAM_BYTES_PER_ENTRY.items():
        if kernel.endswith(suffix):
            return per * entries
    return None


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--rows", type=int, default=20_000_000)
    ap.add_argument("--min-empties", type=int, default=20)
    ap.add_argument("--max-empties", type=int, default=40)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-sample-rows", type=int, default=5_000_000,
                    help="batched workload: rows of the bounded sample the CPU baseline runs")
    ap.add_argument("--lsqr", choices=sorted(LSQ_VARIANTS), default="scaled",
                    help="LSQR/LSMR solves of the single workload reported beside PCG")
    ap.add_argument("--lsqr-max-iterations", type=int, default=20000)
    ap.add_argument("--no-summaries", action="store_true",
                    help="single workload: leave out the short batched and evaluator runs")
    ap.add_argument("--sharded", action="store_true",
                    help="single workload: the row-sharded fit even on one GPU (always with N > 1)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison solve")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--workload", choices=["single", "batched", "evaluator"], default="single",
                    help="single: the 20M-row fit; batched: 60 per-empty-count fits in one batched solve; "
                         "evaluator: one training epoch of the differentiable evaluator")
    ap.add_argument("--eval-rows", type=int, default=8_000_000, help="evaluator: training positions")
    ap.add_argument("--eval-sample-batches", type=int, default=24,
                    help="evaluator: minibatches of the bounded CPU sample")
    ap.add_argument("--problems", type=int, default=60, help="batched: problems (empty counts 1..problems)")
    return ap.parse_args(argv)


def batched_problems(seed: int, problems: int = 60, lo: int = 20_000, hi: int = 1_500_000):
    """Row counts (log-uniform in [lo, hi], seeded) and empty counts 1..problems
    of the batched workload; problem q's positions come from seed 1000 * seed + q."""
    rng = np.random.default_rng(seed)
    rows = np.exp(rng.uniform(np.log(lo), np.log(hi), problems)).astype(np.int64)
    return rows, np.arange(1, problems + 1)


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, flags in rows for i, f in enumerate(flags) if f.lower() == "active"})
        busy = [r[0] for r in rows]
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


def single_config(args) -> dict:
    """The single-fit workload, as both arms name it."""
    return {
        "workload": f"8-pattern expanded fit, {args.rows} rows, empties {args.min_empties}..{args.max_empties}, "
                    f"Jacobi-PCG to rel. normal-eq. residual {args.tol:g}",
        "rows": args.rows, "cols": COLS_8, "nnz_per_row": 64, "nnz": args.rows * 64, "method": "pcg",
        "tol": args.tol, "seed": args.seed,
        "inputs": f"positions {16 * args.rows / 1e6:.0f} MB, index stream {256 * args.rows / 1e9:.2f} GB per "
                  f"product ({'larger' if 256 * args.rows > 126e6 else 'smaller'} than the 126 MB L2)",
    }


COLS_8 = sum(3 ** bin(m).count("1") for m in PATTERNS_8)


# --------------------------------------------------------------------------- ours

def run_ours(args) -> dict | None:
    import torch
    import torch.distributed as dist

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))

    import cassandra_b200 as cb
    from cassandra_b200 import _lib as L

    lib = cb.load()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    seed = args.seed + 7919 * rank
    R = args.rows

    # Inputs, resident in HBM before the timed region (positions 320 MB > L2).
    pos = cb.generate_positions(seed, R, args.min_empties, args.max_empties)
    g = cb.GroupIndexer(PATTERNS_8, "expanded")
    cols, K = g.index_space_size, g.nnz_per_row
    a0 = cb.MatrixCSR.from_positions(g, pos, "rows")
    b = cb.generate_targets(a0, seed)
    torch.cuda.synchronize()
    nnz = R * K

    # ---- roofline of the two sparse products of the mixed solver (FP32, blocked
    # layout), and the same products on the rows layout for reference
    def time_kernel(fn, n=10):
        for _ in range(2):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / n * 1e-3

    x32 = torch.randn(cols, dtype=torch.float32, device="cuda")
    y32 = torch.randn(R, dtype=torch.float32, device="cuda")
    yo = torch.empty(R, dtype=torch.float32, device="cuda")
    xo = torch.empty(cols, dtype=torch.float32, device="cuda")
    kernels = {}

    def measure(a, name, idx_bytes_ax, idx_bytes_aty):
        t_ax = time_kernel(lambda: L.check(lib.cas_spmv(a.handle, L.CAS_F32, C.c_void_p(x32.data_ptr()),
                                                        C.c_void_p(yo.data_ptr()), sp)))
        t_aty = time_kernel(lambda: L.check(lib.cas_spmv_t(a.handle, L.CAS_F32, C.c_void_p(y32.data_ptr()),
                                                           C.c_void_p(xo.data_ptr()), sp)))
        # algorithmic bytes: index stream + the vector written once + the vector read once
        bx = idx_bytes_ax + 4 * R + 4 * cols
        bt = idx_bytes_aty + 4 * R + 4 * cols
        kernels[f"{name}_ax_f32"] = {"seconds": t_ax, "bytes": bx, "gbs": bx / t_ax / 1e9}
        kernels[f"{name}_aty_f32"] = {"seconds": t_aty, "bytes": bt, "gbs": bt / t_aty / 1e9}

    measure(a0, "rows", 4 * nnz, 4 * nnz + 8 * (cols + 1))
    del a0
    torch.cuda.synchronize()
    ab = cb.MatrixCSR.from_positions(g, pos, "blocked")
    measure(ab, "blocked", 2 * nnz, 4 * nnz)
    del ab, x32, y32, yo, xo
    torch.cuda.synchronize()
    # the indexer alone: positions -> uint32 indices [R, K] (16 B read and
    # 4 K B written per position; the 5.1 GB output is larger than L2)
    idx_out = torch.empty((R, K), dtype=torch.int32, device="cuda")
    t_idx = time_kernel(lambda: L.check(lib.cas_index(g.handle, C.c_void_p(pos.data_ptr()), R,
                                                      C.c_void_p(idx_out.data_ptr()), sp)), n=3)
    kernels["index_rows_u32"] = {"seconds": t_idx, "bytes": 16 * R + 4 * nnz, "gbs": (16 * R + 4 * nnz) / t_idx / 1e9}
    del idx_out
    torch.cuda.synchronize()

    opts_mixed = cb.solve_opts("pcg", "mixed", args.tol, 20000, 50, 50)
    opts_plain = cb.solve_opts("pcg", "fp64", args.tol, 20000, 50, 50)
    w = torch.empty(cols, dtype=torch.float64, device="cuda")

    def fit(opts):
        rep = L.SolveReport()
        st = lib.cas_fit_weights_device(g.handle, C.c_void_p(pos.data_ptr()), C.c_void_p(b.data_ptr()), R,
                                        C.byref(opts), C.c_void_p(w.data_ptr()), C.byref(rep), sp)
        if st != L.CAS_OK:
            L.check(st)
        return rep

    for _ in range(args.warmup):
        fit(opts_mixed)
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = lib.cas_kernel_launches()
    # one event between steps (no synchronisation added): the steps' own times
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    reps = []
    for i in range(args.steps):
        reps.append(fit(opts_mixed))
        ev[i + 1].record(stream)
    ev[-1].synchronize()
    torch.cuda.synchronize()
    launches = lib.cas_kernel_launches() - launches0
    clk = clocks.stop()
    elapsed = ev[0].elapsed_time(ev[-1]) * 1e-3
    step_s = [ev[i].elapsed_time(ev[i + 1]) * 1e-3 for i in range(args.steps)]
    if world > 1:
        dist.barrier()
        t = torch.tensor([elapsed], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    per_step = elapsed / args.steps
    mixed = reps[-1]
    solutions = {"mixed_pcg": w.cpu().numpy()}

    # plain FP64 GPU path on the same system, as the fit runs it (rows layout,
    # the reference's structure)
    plain = None
    if not args.no_plain:
        plain = fit(opts_plain)
        solutions["plain_fp64_pcg_rows"] = w.cpu().numpy()

    # the same comparison on one layout: FP64 and mixed PCG solves on one
    # blocked CSR, so the ratio isolates the precision; and LSQR / LSMR
    same_layout, lsq = None, {}
    if not args.no_plain or LSQ_VARIANTS[args.lsqr]:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        ab = cb.MatrixCSR.from_positions(g, pos, "blocked")
        ev1.record(stream)
        ev1.synchronize()
        build_blocked = ev0.elapsed_time(ev1) * 1e-3

        def solve(opts, key):
            rep = L.SolveReport()
            st = lib.cas_solve(ab.handle, C.byref(opts), C.c_void_p(b.data_ptr()), C.c_void_p(w.data_ptr()),
                               C.byref(rep), sp)
            if st not in (L.CAS_OK, L.CAS_ERR_NOT_CONVERGED):
                L.check(st)
            solutions[key] = w.cpu().numpy()
            return {"solve_s": rep.seconds, "iterations": rep.iterations, "refinements": rep.refinements,
                    "rel_residual": rep.rel_residual, "converged": st == L.CAS_OK}

        if not args.no_plain:
            m = solve(opts_mixed, "mixed_pcg_blocked")
            pl = solve(opts_plain, "plain_fp64_pcg_blocked")
            same_layout = {"layout": "blocked", "build_s": build_blocked, "mixed": m, "plain_fp64": pl,
                           "solve_speedup_mixed_vs_plain": pl["solve_s"] / m["solve_s"] if m["solve_s"] else None}
        for method, prec, scaled in LSQ_VARIANTS[args.lsqr]:
            o = cb.solve_opts(method, prec, args.tol, args.lsqr_max_iterations, 50, 100, scale_columns=scaled)
            key = f"{method}_{prec}{'_scaled' if scaled else ''}"
            lsq[key] = solve(o, key)
        del ab
        torch.cuda.synchronize()

    # ---- end to end through the public C ABI with host buffers
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 3))
    e2e_val = None
    pos_h = torch.empty((R, 2), dtype=torch.int64, pin_memory=True)
    pos_h.copy_(pos)
    sc_h = torch.empty(R, dtype=torch.float32, pin_memory=True)
    sc_h.copy_(b.float())
    w_h = torch.empty(cols, dtype=torch.float32, pin_memory=True)
    masks = np.asarray(PATTERNS_8, np.uint64)
    e2e_times = []
    for _ in range(e2e_steps):
        rep = L.SolveReport()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = lib.cas_fit_weights(masks.ctypes.data_as(C.c_void_p), len(masks), L.CAS_INDEX_EXPANDED,
                                 C.c_void_p(pos_h.data_ptr()), C.c_void_p(sc_h.data_ptr()), R, C.byref(opts_mixed),
                                 C.c_void_p(w_h.data_ptr()), C.byref(rep))
        e2e_times.append(time.perf_counter() - t0)
        L.check(st)
    e2e_val = statistics.mean(e2e_times) if e2e_times else None
    if world > 1 and e2e_val is not None:
        t = torch.tensor([e2e_val], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_val = float(t.item())
    e2e = {"value": e2e_val, "unit": "s", "h2d_bytes_per_step": int(pos_h.numel() * 8 + sc_h.numel() * 4),
           "d2h_bytes_per_step": int(w_h.numel() * 4), "steps": e2e_steps}

    peak, peak_kind = measured_peaks()
    blocked = {k: v for k, v in kernels.items() if k.startswith("blocked")}
    dom = max(blocked, key=lambda k: blocked[k]["seconds"])
    ach = kernels[dom]["gbs"]

    # ---- the reference's own code on the host cores, on the same system: the
    # CPU baseline (the whole workload, one step) and the oracle check of
    # every solution above
    cpu, check = None, None
    pos_host = pos.cpu().numpy().view(np.uint64)
    b_host = b.cpu().numpy()
    del pos, b, pos_h, sc_h, w_h
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, check = reference_check(args, pos_host, b_host, solutions)

    summaries = {}
    if world == 1 and not args.no_summaries:
        import gc

        gc.collect()
        torch.cuda.empty_cache()
        summaries["batched"] = compact(run_ours_batched(summary_args(args)))
        gc.collect()
        torch.cuda.empty_cache()
        summaries["evaluator"] = compact(run_ours_evaluator(summary_args(args)))
        gc.collect()
        torch.cuda.empty_cache()
        summaries["config0"] = run_config0(args)

    result = {
        "metric": METRIC,
        "value": per_step,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": per_step * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 products / f64 scalars",
        "data": "synthetic (seeded random-play positions, seeded targets)",
        "config": single_config(args),
        "precision": "mixed (FP32 products on the blocked layout, FP64 compensated scalars, reliable updating)",
        "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "breakdown": {
            "step_s": step_s, "build_s_steps": [r.setup_seconds for r in reps],
            "build_s": mixed.setup_seconds, "solve_s": mixed.seconds, "iterations": mixed.iterations,
            "refinements": mixed.refinements, "rel_residual": mixed.rel_residual,
        },
        "plain_fp64": None if plain is None else {
            "layout": "rows", "step_s": plain.setup_seconds + plain.seconds, "solve_s": plain.seconds,
            "iterations": plain.iterations, "rel_residual": plain.rel_residual,
            "solve_speedup_mixed_vs_plain": plain.seconds / mixed.seconds if mixed.seconds else None,
        },
        "same_layout": same_layout,
        "least_squares": lsq or None,
        "oracle_check": check,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "peak_kind": peak_kind, "traffic": ncu_traffic(dom, nnz),
                     "traffic_unit": "bytes per launch, scaled from ncu at 2M rows"},
        "kernels": kernels,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clk,
        "cpu_baseline": cpu,
        "summaries": summaries or None,
    }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result if rank == 0 else None


def run_ours_sharded(args) -> dict | None:
    """The single workload on N GPUs as one fit sharded by rows: rank k holds
    the rows of its block range of the 20M-row system (positions from the
    seeded generator at those row numbers, the system's targets for them),
    and every step builds its blocked CSR and runs the row-sharded mixed PCG
    (cassandra_b200.parallel: one all-reduce of cols + 1 doubles per
    iteration, FP64 residual replacement at chunk boundaries) to the
    tolerance.  Total work is fixed: strong scaling."""
    import datetime

    import torch
    import torch.distributed as dist

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world == 1:  # --sharded on one GPU: a process group of one rank
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29511")
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    import cassandra_b200 as cb
    from cassandra_b200 import parallel as par

    lib = cb.load()
    stream = torch.cuda.current_stream()
    R = args.rows
    lo, hi = par.split_rows(R, world, rank, int(lib.cas_block_rows()))
    n = hi - lo
    g = cb.GroupIndexer(PATTERNS_8, "expanded")
    pos_h = torch.from_numpy(cb.generate_positions_host(args.seed, lo, n, args.min_empties, args.max_empties)
                             .view(np.int64).reshape(n, 2)).pin_memory()
    pos = pos_h.to("cuda")
    b = cb.generate_targets(cb.MatrixCSR.from_positions(g, pos, "rows"), args.seed, first_row=lo)
    torch.cuda.synchronize()

    def step():
        a = cb.MatrixCSR.from_positions(g, pos, "blocked")
        return par.sharded_pcg(par.GpuShard(a, b, "mixed"), tol=args.tol, max_iterations=20000)

    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(local)
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = lib.cas_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    results = [step() for _ in range(args.steps)]
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    launches = lib.cas_kernel_launches() - launches0
    clk = clocks.stop()
    t = torch.tensor([e0.elapsed_time(e1) * 1e-3], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    per_step = float(t.item()) / args.steps
    last = results[-1]

    # end to end: the rank's positions and targets from pinned host memory,
    # the fit, the weights back
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 2))
    b_h = b.cpu().pin_memory()
    w_h = torch.empty(COLS_8, dtype=torch.float64).pin_memory()
    times = []
    for _ in range(e2e_steps):
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        p_d, b_d = pos_h.to("cuda", non_blocking=True), b_h.to("cuda", non_blocking=True)
        a = cb.MatrixCSR.from_positions(g, p_d, "blocked")
        res = par.sharded_pcg(par.GpuShard(a, b_d, "mixed"), tol=args.tol, max_iterations=20000)
        w_h.copy_(res.x)
        times.append(time.perf_counter() - t0)
    te = torch.tensor([statistics.mean(times)], dtype=torch.float64, device="cuda")
    dist.all_reduce(te, op=dist.ReduceOp.MAX)
    peak, peak_kind = measured_peaks()
    result = {
        "metric": METRIC, "value": per_step, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": False, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32 products / f64 scalars",
        "data": "synthetic (seeded random-play positions, seeded targets)",
        "config": single_config(args),
        "precision": "mixed (FP32 products, FP64 replicated state, FP64 residual replacement on a 1e3 drop or "
                     "every 50 iterations)",
        "parallelism": f"row-sharded x{world}: one all-reduce of {COLS_8 + 1} doubles per iteration (NCCL)",
        "breakdown": {"iterations": last.iterations, "replacements": last.replacements,
                      "allreduces": last.allreduces, "rel_residual": last.rel_residual,
                      "rows_per_rank": n},
        "roofline": None, "peak_hbm_gbs": peak, "peak_kind": peak_kind,
        "e2e": {"value": float(te.item()), "unit": "s", "h2d_bytes_per_step": int(n * 16 + n * 8),
                "d2h_bytes_per_step": COLS_8 * 8, "steps": e2e_steps},
        "gpu_launches": int(launches), "clocks": clk, "cpu_baseline": None,
    }
    dist.barrier()
    dist.destroy_process_group()
    return result if rank == 0 else None


# LSQR / LSMR solves of the single workload: (method, precision, column scaling)
LSQ_VARIANTS = {
    "none": [],
    "scaled": [("lsqr", "mixed", True), ("lsqr", "fp64", True)],
    "all": [("lsqr", "mixed", True), ("lsqr", "fp64", True), ("lsqr", "mixed", False), ("lsqr", "fp64", False),
            ("lsmr", "mixed", True), ("lsmr", "mixed", False)],
}


def summary_args(args):
    """A short run of another workload for the default line: 2 steps after
    3 warm-ups, no sequential plain comparison, no end-to-end pass, a smaller
    CPU sample."""
    d = dict(vars(args))
    d.update(steps=2, warmup=3, no_plain=True, e2e_steps=0, cpu_sample_rows=1_000_000, eval_sample_batches=8)
    return argparse.Namespace(**d)


def compact(res: dict | None) -> dict | None:
    if res is None:
        return None
    keep = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "config", "roofline", "kernels",
            "gpu_launches", "cpu_baseline", "clocks", "least_squares")
    out = {k: res[k] for k in keep if k in res}
    br = res.get("breakdown", {})
    out["breakdown"] = {k: v for k, v in br.items() if k != "per_problem"}
    return out


def run_ours_batched(args) -> dict | None:
    """60 per-empty-count fits (empty counts 1..60, rows log-uniform in
    [20k, 1.5M], seeded) as one step: batched layout build + one batched
    mixed-precision PCG to 1e-8 for every problem.  The plain FP64 GPU path
    fits the same problems one after another on the rows layout; the LSQR
    variants of --lsqr fit them with one solver per problem, run together."""
    import torch
    import torch.distributed as dist

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    import cassandra_b200 as cb
    from cassandra_b200 import _lib as L

    lib = cb.load()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    seed = args.seed + 7919 * rank
    rows, empties = batched_problems(seed, args.problems)
    R = int(rows.sum())
    pos = torch.cat([cb.generate_positions(1000 * seed + q, int(n), int(e), int(e))
                     for q, (n, e) in enumerate(zip(rows, empties))])
    g = cb.GroupIndexer(PATTERNS_8, "expanded")
    cols, K = g.index_space_size, g.nnz_per_row
    P = len(rows)
    a0 = cb.MatrixCSR.from_positions_batched(g, pos, rows)
    b = cb.generate_targets(a0, seed)
    torch.cuda.synchronize()
    nnz = R * K

    # roofline of the FP32 products on the batched layout (all problems active)
    def time_kernel(fn, n=10):
        for _ in range(2):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / n * 1e-3

    x32 = torch.randn(P * cols, dtype=torch.float32, device="cuda")
    y32 = torch.randn(R, dtype=torch.float32, device="cuda")
    yo = torch.empty(R, dtype=torch.float32, device="cuda")
    xo = torch.empty(P * cols, dtype=torch.float32, device="cuda")
    t_ax = time_kernel(lambda: L.check(lib.cas_spmv(a0.handle, L.CAS_F32, C.c_void_p(x32.data_ptr()),
                                                    C.c_void_p(yo.data_ptr()), sp)))
    t_aty = time_kernel(lambda: L.check(lib.cas_spmv_t(a0.handle, L.CAS_F32, C.c_void_p(y32.data_ptr()),
                                                       C.c_void_p(xo.data_ptr()), sp)))
    bx = 2 * nnz + 4 * R + 4 * P * cols
    bt = 4 * nnz + 4 * R + 4 * P * cols
    kernels = {"batched_ax_f32": {"seconds": t_ax, "bytes": bx, "gbs": bx / t_ax / 1e9},
               "batched_aty_f32": {"seconds": t_aty, "bytes": bt, "gbs": bt / t_aty / 1e9}}
    schedules = a0.schedules()
    del x32, y32, yo, xo, a0
    torch.cuda.synchronize()

    opts_mixed = cb.solve_opts("pcg", "mixed", args.tol, 20000, 50, 50)
    opts_plain = cb.solve_opts("pcg", "fp64", args.tol, 20000, 50, 50)
    w = torch.empty(P * cols, dtype=torch.float64, device="cuda")
    rows_c = np.ascontiguousarray(rows, dtype=np.int64)

    def fit_batched():
        reps = (L.SolveReport * P)()
        st = lib.cas_fit_weights_batched_device(g.handle, C.c_void_p(pos.data_ptr()), C.c_void_p(b.data_ptr()),
                                                rows_c.ctypes.data_as(C.c_void_p), P, C.byref(opts_mixed),
                                                C.c_void_p(w.data_ptr()), reps, sp)
        if st != L.CAS_OK:
            L.check(st)
        return reps

    for _ in range(args.warmup):
        fit_batched()
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = lib.cas_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    reps = [fit_batched() for _ in range(args.steps)]
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    launches = lib.cas_kernel_launches() - launches0
    clk = clocks.stop()
    elapsed = e0.elapsed_time(e1) * 1e-3
    if world > 1:
        dist.barrier()
        t = torch.tensor([elapsed], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    per_step = elapsed / args.steps
    last = reps[-1]
    its = [r.iterations for r in last]

    # plain FP64 GPU path: the problems fitted one after another (rows layout)
    plain = None
    if not args.no_plain:
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        r0 = np.concatenate([[0], np.cumsum(rows)])
        plain_its, plain_rel, plain_t = [], [], []
        wq = torch.empty(cols, dtype=torch.float64, device="cuda")
        for q in range(P):
            rep = L.SolveReport()
            st = lib.cas_fit_weights_device(g.handle, C.c_void_p(pos[r0[q]:r0[q + 1]].data_ptr()),
                                            C.c_void_p(b[r0[q]:r0[q + 1]].data_ptr()), int(rows[q]),
                                            C.byref(opts_plain), C.c_void_p(wq.data_ptr()), C.byref(rep), sp)
            if st != L.CAS_OK:
                L.check(st)
            plain_its.append(rep.iterations)
            plain_rel.append(rep.rel_residual)
            plain_t.append(rep.setup_seconds + rep.seconds)
        p1.record(stream)
        p1.synchronize()
        plain = {"step_s": p0.elapsed_time(p1) * 1e-3, "iterations_max": max(plain_its),
                 "iterations_sum": int(sum(plain_its)), "rel_residual_max": max(plain_rel),
                 "speedup_batched_mixed_vs_sequential_plain": p0.elapsed_time(p1) * 1e-3 / per_step,
                 "per_problem": [[int(i), round(t, 5)] for i, t in zip(plain_its, plain_t)]}

    # the same fits by LSQR (--lsqr variants), one solver per problem, all
    # run together on their own streams (cas_fit_weights_batched_device with
    # method LSQR): one untimed warm-up, then one step on the host clock (the
    # call returns when every problem has finished)
    least_squares = {}
    for method, prec, scaled in LSQ_VARIANTS[args.lsqr]:
        o = cb.solve_opts(method, prec, args.tol, args.lsqr_max_iterations, 50, 100, scale_columns=scaled)
        wl = torch.empty(P * cols, dtype=torch.float64, device="cuda")

        def fit_lsq():
            lreps = (L.SolveReport * P)()
            st = lib.cas_fit_weights_batched_device(g.handle, C.c_void_p(pos.data_ptr()), C.c_void_p(b.data_ptr()),
                                                    rows_c.ctypes.data_as(C.c_void_p), P, C.byref(o),
                                                    C.c_void_p(wl.data_ptr()), lreps, sp)
            if st not in (L.CAS_OK, L.CAS_ERR_NOT_CONVERGED):
                L.check(st)
            return st, lreps

        fit_lsq()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st, lreps = fit_lsq()
        torch.cuda.synchronize()
        least_squares[f"{method}_{prec}{'_scaled' if scaled else ''}"] = {
            "step_s": time.perf_counter() - t0, "converged": st == L.CAS_OK,
            "iterations_max": max(r.iterations for r in lreps),
            "iterations_sum": int(sum(r.iterations for r in lreps)),
            "rel_residual_max": max(r.rel_residual for r in lreps)}
        del wl

    # end to end through the public C ABI with host buffers
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 3))
    pos_h = torch.empty((R, 2), dtype=torch.int64, pin_memory=True)
    pos_h.copy_(pos)
    sc_h = torch.empty(R, dtype=torch.float32, pin_memory=True)
    sc_h.copy_(b.float())
    w_h = torch.empty(P * cols, dtype=torch.float32, pin_memory=True)
    masks = np.asarray(PATTERNS_8, np.uint64)
    e2e_times = []
    for _ in range(e2e_steps):
        hreps = (L.SolveReport * P)()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = lib.cas_fit_weights_batched(masks.ctypes.data_as(C.c_void_p), len(masks), L.CAS_INDEX_EXPANDED,
                                         C.c_void_p(pos_h.data_ptr()), C.c_void_p(sc_h.data_ptr()),
                                         rows_c.ctypes.data_as(C.c_void_p), P, C.byref(opts_mixed),
                                         C.c_void_p(w_h.data_ptr()), hreps)
        e2e_times.append(time.perf_counter() - t0)
        L.check(st)
    e2e_val = statistics.mean(e2e_times) if e2e_times else None

    peak, peak_kind = measured_peaks()
    dom = max(kernels, key=lambda k: kernels[k]["seconds"])
    ach = kernels[dom]["gbs"]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_batched(args, seed, rows, empties)
    result = {
        "metric": METRIC, "value": per_step, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 products / f64 scalars",
        "data": "synthetic (seeded random-play positions per empty count, seeded targets)",
        "config": {
            "workload": f"{P} per-empty-count 8-pattern expanded fits (empties 1..{P}, rows log-uniform in "
                        f"[20k, 1.5M], {R} rows in total), one batched mixed Jacobi-PCG to rel. normal-eq. "
                        f"residual {args.tol:g} per problem",
            "problems": P, "rows": R, "cols_per_problem": cols, "nnz_per_row": K, "nnz": nnz,
            "rows_min": int(rows.min()), "rows_max": int(rows.max()), "precision": "mixed", "tol": args.tol,
            "l2": "inputs larger than L2", "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        },
        "breakdown": {"build_s": last[0].setup_seconds, "solve_s": last[0].seconds,
                      "iterations_max": max(its), "iterations_min": min(its),
                      "rel_residual_max": max(r.rel_residual for r in last),
                      "per_problem": [[int(n), int(e), int(r.iterations), int(r.refinements)]
                                      for n, e, r in zip(rows, empties, last)]},
        "plain_fp64": plain,
        "least_squares": least_squares or None,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "peak_kind": peak_kind, "traffic": ncu_traffic(dom, nnz),
                     "traffic_unit": "bytes per launch, scaled from ncu at 2M rows"},
        "kernels": kernels, "aty_schedules": schedules,
        "e2e": {"value": e2e_val, "unit": "s", "h2d_bytes_per_step": int(pos_h.numel() * 8 + sc_h.numel() * 4),
                "d2h_bytes_per_step": int(w_h.numel() * 4), "steps": e2e_steps},
        "gpu_launches": int(launches), "clocks": clk, "cpu_baseline": cpu,
    }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result if rank == 0 else None


CONFIG0_METRIC = "seconds for FitWeights(pattern, positions, 200): index, CSR, Jacobi, 200 PCG iterations"
PATTERNS_5 = PATTERNS_8[:5]


def run_config0(args) -> dict:
    """The reference's CPU-runnable case: 100,000 positions at exactly 30
    empties, the 5-pattern set expanded (150,903 columns, 40 entries per
    row), targets by the seeded recipe, Jacobi-PCG from x0 = 0 for exactly
    200 iterations (FitWeights(pattern, positions, 200),
    PatternFit/PatternFit.cpp:7-39).  GPU: one step = cas_fit_weights_device
    (indexing, the layout, Jacobi and the 200 iterations) on the plain FP64
    path (rows layout) and on the mixed path, CUDA events; e2e through
    cas_fit_weights with host buffers; CPU: the reference compiled from its
    sources (FP32 as shipped), indexing and the 200 iterations on the host
    cores."""
    import torch

    import cassandra_b200 as cb
    import oracle
    from cassandra_b200 import _lib as L

    lib = cb.load()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    rows, iters, seed = 100_000, 200, args.seed
    pos = cb.generate_positions(seed, rows, 30, 30)
    g = cb.GroupIndexer(PATTERNS_5, "expanded")
    cols, K = g.index_space_size, g.nnz_per_row
    b = cb.generate_targets(cb.MatrixCSR.from_positions(g, pos, "rows"), seed)
    w = torch.empty(cols, dtype=torch.float64, device="cuda")
    out = {}
    for precision in ("fp64", "mixed"):
        opts = cb.solve_opts("pcg", precision, 0.0, iters, 50, 50)

        def step():
            rep = L.SolveReport()
            L.check(lib.cas_fit_weights_device(g.handle, C.c_void_p(pos.data_ptr()), C.c_void_p(b.data_ptr()), rows,
                                               C.byref(opts), C.c_void_p(w.data_ptr()), C.byref(rep), sp))
            return rep

        for _ in range(2):
            step()
        # an event between steps: the steps' own device times; this step is
        # launch-bound (200 iterations of small kernels), so the median of 5
        # is reported beside all five
        n = 5
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(n + 1)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        for i in range(n):
            rep = step()
            ev[i + 1].record(stream)
        ev[-1].synchronize()
        steps = [ev[i].elapsed_time(ev[i + 1]) * 1e-3 for i in range(n)]
        out[precision] = {"step_s": statistics.median(steps), "step_s_all": steps, "iterations": int(rep.iterations),
                          "rel_residual": rep.rel_residual}
    # end to end with host buffers (plain FP64 path)
    pos_h = np.ascontiguousarray(pos.cpu().numpy().view(np.uint64))
    sc_h = np.ascontiguousarray(b.cpu().numpy().astype(np.float32))
    w_h = np.empty(cols, np.float32)
    masks = np.asarray(PATTERNS_5, np.uint64)
    opts = cb.solve_opts("pcg", "fp64", 0.0, iters, 50, 50)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rep = L.SolveReport()
    L.check(lib.cas_fit_weights(masks.ctypes.data_as(C.c_void_p), len(masks), L.CAS_INDEX_EXPANDED,
                                pos_h.ctypes.data_as(C.c_void_p), sc_h.ctypes.data_as(C.c_void_p), rows,
                                C.byref(opts), w_h.ctypes.data_as(C.c_void_p), C.byref(rep)))
    e2e = time.perf_counter() - t0
    # the reference on the host cores: its indexing (A_Indexer recipe) and its
    # FP32 PCG, 200 iterations
    cpu = {"value": None, "unit": "s", "cores": _threads(), "kind": "reference",
           "sample": f"the whole workload: reference indexing + FP32 PCG, {iters} iterations"}
    if not args.no_cpu_baseline:
        try:
            ref = oracle.ref_lib()
        except (OSError, FileNotFoundError) as e:
            cpu["sample"] = f"reference library unavailable: {e}"
        else:
            ref.ref_expanded_index.restype = None
            ref.ref_expanded_index.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p]
            idx = np.empty((rows, K), np.uint32)
            x = np.empty(cols, np.float32)
            res = C.c_float()
            t0 = time.perf_counter()
            ref.ref_expanded_index(masks.ctypes.data_as(C.c_void_p), len(masks), pos_h.ctypes.data_as(C.c_void_p),
                                   rows, idx.ctypes.data_as(C.c_void_p))
            ref.ref_pcg(K, rows, cols, idx.ctypes.data_as(C.c_void_p), sc_h.ctypes.data_as(C.c_void_p), iters,
                        x.ctypes.data_as(C.c_void_p), C.byref(res))
            cpu["value"] = time.perf_counter() - t0
    return {
        "metric": CONFIG0_METRIC, "value": out["fp64"]["step_s"], "unit": "s", "higher_is_better": False,
        "timing": "median of 5 steps, CUDA events between steps (all five in step_s_all)",
        "config": {"workload": f"5-pattern expanded fit, {rows} positions at 30 empties, Jacobi-PCG x0 = 0, "
                               f"{iters} iterations", "rows": rows, "cols": cols, "nnz_per_row": K},
        "plain_fp64": out["fp64"], "mixed": out["mixed"], "e2e": {"value": e2e, "unit": "s"},
        "cpu_baseline": cpu,
    }


EVAL_METRIC = "differentiable evaluator: seconds per training epoch (Huber+L2, Adam, batch 65536)"
EVAL_EMPTIES = (10, 50)
EVAL_BATCH = 65536
EVAL_LR, EVAL_L2, EVAL_DELTA = 1e-2, 1e-4, 4.0


def eval_config(rows: int) -> dict:
    return {"workload": f"differentiable evaluator, 8-pattern expanded, {rows} positions (empties "
                        f"{EVAL_EMPTIES[0]}..{EVAL_EMPTIES[1]}), one epoch of Adam (lr {EVAL_LR:g}) on mean "
                        f"Huber (delta {EVAL_DELTA:g}) + L2 {EVAL_L2:g} over shuffled {EVAL_BATCH}-row minibatches",
            "rows": rows, "batch": EVAL_BATCH, "l2": "inputs larger than L2 (CSR 3 GB; each kernel pass 1-2 GB)"}


def run_ours_evaluator(args) -> dict | None:
    import torch
    import torch.distributed as dist

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))

    import cassandra_b200 as cb
    from cassandra_b200 import _lib as L
    from cassandra_b200 import evaluator as ev

    lib = cb.load()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    seed = args.seed + 7919 * rank
    R = args.eval_rows

    pos = cb.generate_positions(seed, R, *EVAL_EMPTIES)
    model = ev.PatternEvaluator(PATTERNS_8, pos, "expanded")
    cols, K = model.indexer.index_space_size, model.indexer.nnz_per_row
    target = cb.generate_targets(model.csr, seed).float()
    trainer = ev.Trainer(model, target, batch=EVAL_BATCH, lr=EVAL_LR, l2=EVAL_L2, delta=EVAL_DELTA, seed=seed)
    batches = trainer.batches
    torch.cuda.synchronize()

    # ---- the two kernels, every minibatch once per pass (a pass reads 1-2 GB > L2)
    w = model.weight.detach()
    g = torch.randn(max(r1 - r0 for r0, r1 in batches), dtype=torch.float32, device="cuda")
    score = torch.empty_like(g)
    grad = torch.empty(cols, dtype=torch.float32, device="cuda")

    def one_pass(fn):
        for r0, r1 in batches:
            L.check(fn(model.csr.handle, r0, r1))

    fwd = lambda h, r0, r1: lib.cas_eval_forward(h, r0, r1, C.c_void_p(w.data_ptr()), C.c_void_p(score.data_ptr()), sp)
    bwd = lambda h, r0, r1: lib.cas_eval_backward(h, r0, r1, C.c_void_p(g.data_ptr()), C.c_void_p(grad.data_ptr()), sp)
    kernels = {}
    for name, fn, idx_bytes in (("eval_forward_f32", fwd, 2), ("eval_backward_f32", bwd, 4)):
        one_pass(fn)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(3):
            one_pass(fn)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1) * 1e-3 / (3 * len(batches))
        by = (idx_bytes * K + 4) * R / len(batches) + 4 * cols  # per launch: entries + rows + the C-vector
        kernels[name] = {"seconds": t, "bytes": by, "gbs": by / t / 1e9}
    # the whole training step (three kernels) eagerly, every minibatch once
    # per pass, on scratch weights and moments
    ws, ms, vs = w.clone(), torch.zeros_like(w), torch.zeros_like(w)
    st = torch.zeros((), dtype=torch.int64, device="cuda")
    ls = torch.zeros((), dtype=torch.float64, device="cuda")
    step_fn = lambda h, r0, r1: lib.cas_eval_adam_step(
        h, r0, r1, C.c_void_p(target[r0:r1].data_ptr()), C.c_void_p(ws.data_ptr()), C.c_void_p(ms.data_ptr()),
        C.c_void_p(vs.data_ptr()), C.c_void_p(st.data_ptr()), C.c_void_p(ls.data_ptr()), C.byref(trainer.opts), sp)
    one_pass(step_fn)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(3):
        one_pass(step_fn)
    e1.record(stream)
    e1.synchronize()
    t_step = e0.elapsed_time(e1) * 1e-3 / (3 * len(batches))
    by_step = (6 * K + 4) * R / len(batches) + 24 * cols  # A16 + G32 + targets; w, m, v read and written
    train_step = {"seconds": t_step, "bytes": by_step, "gbs": by_step / t_step / 1e9, "kernels": 3}
    del g, score, grad, ws, ms, vs, st, ls

    for _ in range(args.warmup):
        trainer.epoch()
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = lib.cas_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    losses = [trainer.epoch() for _ in range(args.steps)]
    e1.record(stream)
    e1.synchronize()
    launches_host = lib.cas_kernel_launches() - launches0
    clk = clocks.stop()
    elapsed = e0.elapsed_time(e1) * 1e-3
    if world > 1:
        dist.barrier()
        t = torch.tensor([elapsed], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    per_epoch = elapsed / args.steps
    # graph replays launch the captured kernels without the host counter:
    # three of ours (forward with the loss, A'y partials, Adam epilogue) per minibatch
    launches = launches_host + 3 * len(batches) * args.steps

    # ---- end to end through the public API with host buffers: copy the
    # positions and targets in, build the model, one epoch, read the loss
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 2))
    pos_h = torch.empty((R, 2), dtype=torch.int64, pin_memory=True)
    pos_h.copy_(pos)
    tg_h = torch.empty(R, dtype=torch.float32, pin_memory=True)
    tg_h.copy_(target)
    del trainer, model, pos, target
    torch.cuda.synchronize()
    e2e_times = []
    for _ in range(e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        p_d = pos_h.to("cuda", non_blocking=True)
        t_d = tg_h.to("cuda", non_blocking=True)
        m = ev.PatternEvaluator(PATTERNS_8, p_d, "expanded")
        tr = ev.Trainer(m, t_d, batch=EVAL_BATCH, lr=EVAL_LR, l2=EVAL_L2, delta=EVAL_DELTA, seed=seed)
        tr.epoch()  # ends with the loss read
        e2e_times.append(time.perf_counter() - t0)
        del tr, m, p_d, t_d
    e2e_val = statistics.mean(e2e_times) if e2e_times else None
    if world > 1 and e2e_val is not None:
        t = torch.tensor([e2e_val], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_val = float(t.item())

    peak, peak_kind = measured_peaks()
    dom = max(kernels, key=lambda k: kernels[k]["seconds"])
    ach = kernels[dom]["gbs"]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_evaluator(args, seed, len(batches))
    result = {
        "metric": EVAL_METRIC, "value": per_epoch, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_epoch * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random-play positions, seeded targets; random-init weights)",
        "config": {**eval_config(R), "cols": cols, "nnz_per_row": K, "minibatches": len(batches),
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "breakdown": {"epoch_losses": losses, "batch_step_us": per_epoch / len(batches) * 1e6,
                      "graphs": len(batches), "train_step_eager": train_step},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "peak_kind": peak_kind, "traffic": None},
        "kernels": kernels,
        "e2e": {"value": e2e_val, "unit": "s", "h2d_bytes_per_step": int(pos_h.numel() * 8 + tg_h.numel() * 4),
                "d2h_bytes_per_step": 4, "steps": e2e_steps,
                "includes": "H2D of positions and targets, model build (indexing, blocked CSR), graph capture, "
                            "one epoch, loss read"},
        "gpu_launches": int(launches), "clocks": clk, "cpu_baseline": cpu,
    }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result if rank == 0 else None


# ---------------------------------------------------------------- CPU reference

class ReferenceSystem:
    """One fit's system on the host, run with the reference's own code: its
    A_Indexer recipe over FastIndex/Flipped* for the expanded layout
    (oracle/ref/ref_driver.cpp) and its Math/ PCG retyped to FP64
    (oracle/ref/ref64_driver.cpp, FitWeights' solve, PatternFit/PatternFit.cpp:
    24-32), to a relative normal-equation residual of tol.  Positions are
    given, or made by the oracle's restatement of the seeded generator (this
    process never loads the CUDA library); targets likewise."""

    def __init__(self, seed: int, rows: int, min_e: int, max_e: int, pos: np.ndarray | None = None,
                 b: np.ndarray | None = None, first: int = 0):
        import oracle

        self.ref, self.ref64 = oracle.ref_lib(), oracle.ref64_lib()
        self.ref.ref_expanded_index.restype = None
        self.ref.ref_expanded_index.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p]
        self.rows = rows
        self.masks = np.asarray(PATTERNS_8, np.uint64)
        self.cols = COLS_8
        self.pos = np.ascontiguousarray(pos if pos is not None else
                                        oracle.generate_positions(seed, first, rows, min_e, max_e), dtype=np.uint64)
        self.idx = np.empty((rows, 64), np.uint32)
        self.index()
        self.b = b if b is not None else oracle.generate_targets(self.idx, self.cols, seed)[0]

    def index(self) -> float:
        t0 = time.perf_counter()
        self.ref.ref_expanded_index(self.masks.ctypes.data_as(C.c_void_p), len(self.masks),
                                    self.pos.ctypes.data_as(C.c_void_p), self.rows,
                                    self.idx.ctypes.data_as(C.c_void_p))
        return time.perf_counter() - t0

    def run(self, tol: float) -> dict:
        """One step: indexing and the FP64 PCG (Jacobi set-up included; its
        residual checks every 10 iterations excluded from the time)."""
        t_index = self.index()
        x = np.empty(self.cols)
        rel, sec = np.zeros(1), np.zeros(1)
        it = self.ref64.ref64_pcg(64, self.rows, self.cols, self.idx.ctypes.data_as(C.c_void_p),
                                  self.b.ctypes.data_as(C.c_void_p), 20000, tol, 10, x.ctypes.data_as(C.c_void_p),
                                  rel.ctypes.data_as(C.c_void_p), sec.ctypes.data_as(C.c_void_p))
        return {"index_s": t_index, "solve_s": float(sec[0]), "step_s": t_index + float(sec[0]),
                "iterations": int(it), "rel_residual": float(rel[0]), "x": x}

    def check(self, xs: list[np.ndarray]) -> tuple[list[float], np.ndarray]:
        """FP64 normal residuals of the given solutions with the reference's
        products, and the mask of columns with entries."""
        n = len(xs)
        flat = np.ascontiguousarray(np.stack(xs) if n else np.zeros((0, self.cols)), dtype=np.float64)
        out = np.empty(max(n, 1))
        hit = np.empty(self.cols, np.uint8)
        self.ref64.ref64_check(64, self.rows, self.cols, self.idx.ctypes.data_as(C.c_void_p),
                               self.b.ctypes.data_as(C.c_void_p), n, flat.ctypes.data_as(C.c_void_p),
                               out.ctypes.data_as(C.c_void_p), hit.ctypes.data_as(C.c_void_p))
        return [float(v) for v in out[:n]], hit.astype(bool)


def _threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))


def reference_check(args, pos: np.ndarray, b: np.ndarray, solutions: dict) -> tuple[dict, dict]:
    """The reference's FP64 PCG on the benchmarked system (the CPU baseline,
    one full step) and the check of the device's solutions against it: each
    solution's FP64 normal-equation residual with the reference's products,
    and its largest weight difference from the reference's solution on the
    columns with entries (x0 = 0 and the Jacobi preconditioner in both fix
    the gauge of the rank-deficient system)."""
    try:
        import oracle

        if not oracle.ref_available():
            return ({"value": None, "unit": "s", "cores": _threads(), "kind": "reference",
                     "sample": "unavailable: oracle/_ref not built"}, None)
    except Exception as e:  # pragma: no cover
        return ({"value": None, "unit": "s", "cores": _threads(), "kind": "reference", "sample": f"error {e}"},
                None)
    sysm = ReferenceSystem(args.seed, args.rows, args.min_empties, args.max_empties, pos=pos, b=b)
    r = sysm.run(args.tol)
    names = list(solutions)
    rels, hit = sysm.check([solutions[k] for k in names] + [r["x"]])
    xr = r["x"][hit]
    scale = float(np.abs(xr).max()) if xr.size else 1.0
    check = {"reference": {"method": "reference Math/ PCG retyped to FP64, Jacobi, x0 = 0",
                           "iterations": r["iterations"], "rel_residual_fp64": rels[-1]},
             "hit_cols": int(hit.sum()), "cols": int(hit.size)}
    for k, rel in zip(names, rels):
        d = np.abs(solutions[k][hit] - xr)
        check[k] = {"rel_residual_fp64": rel, "max_weight_err_hit": float(d.max()) if d.size else 0.0,
                    "max_weight_err_hit_rel": float(d.max()) / scale if d.size else 0.0}
    cpu = {"value": r["step_s"], "unit": "s", "cores": _threads(), "kind": "reference",
           "sample": f"the whole workload ({args.rows} rows), one step on the same system as the GPU arm: reference "
                     f"A_Indexer recipe (FastIndex/Flipped*) {r['index_s']:.2f} s + reference Math/ PCG retyped to "
                     f"FP64 to {args.tol:g}, {r['iterations']} iterations, {r['solve_s']:.2f} s "
                     f"(rel {r['rel_residual']:.2e}); OpenMP threads {_threads()}"}
    return cpu, check


def cpu_baseline_batched(args, seed: int, rows, empties) -> dict | None:
    """The reference fitting the batched workload's problems one after another
    (its training loop's order), on a bounded sample: the first problems in
    order until about cpu_sample_rows rows, time scaled by total rows.
    Positions are the batched workload's (per-problem streams); targets follow
    the same recipe from per-problem streams."""
    try:
        import oracle

        if not oracle.ref_available():
            return {"value": None, "unit": "s", "cores": _threads(), "kind": "reference",
                    "sample": "unavailable: oracle/_ref not built"}
    except Exception as e:  # pragma: no cover
        return {"value": None, "unit": "s", "cores": _threads(), "kind": "reference", "sample": f"error {e}"}
    total, done_rows, t, its = int(np.sum(rows)), 0, 0.0, []
    for q, (n, e) in enumerate(zip(rows, empties)):
        if done_rows >= args.cpu_sample_rows:
            break
        s = ReferenceSystem(1000 * seed + q, int(n), int(e), int(e)).run(args.tol)
        t += s["step_s"]
        its.append(s["iterations"])
        done_rows += int(n)
    return {"value": t * total / done_rows, "unit": "s", "cores": _threads(), "kind": "reference",
            "sample": f"first {len(its)} of {len(rows)} problems ({done_rows} of {total} rows), each: reference "
                      f"indexing + FP64 PCG to {args.tol:g} ({min(its)}..{max(its)} iterations); time scaled by rows "
                      f"x{total / done_rows:.3g}"}


def cpu_baseline_evaluator(args, seed: int, batches_per_epoch: int) -> dict | None:
    """The same training step on the host cores with the reference's own
    products (MatrixCSR * Vector and Vector * MatrixCSR, Math/MatrixCSR.cpp:
    49-87, OpenMP) on a bounded sample of minibatches, the loss, its
    gradient and Adam in numpy; the time per minibatch scaled to an epoch.
    Indexing and the per-minibatch MatrixCSR are prepared untimed, as the
    GPU arm prepares its CSR before the epoch."""
    try:
        import oracle

        if not oracle.ref_available():
            return {"value": None, "unit": "s", "cores": _threads(), "kind": "reference",
                    "sample": "unavailable: oracle/_ref not built"}
    except Exception as e:  # pragma: no cover
        return {"value": None, "unit": "s", "cores": _threads(), "kind": "reference", "sample": f"error {e}"}
    nb = max(1, min(args.eval_sample_batches, batches_per_epoch))
    rows = nb * EVAL_BATCH
    smp = ReferenceSystem(seed, rows, *EVAL_EMPTIES)
    lib, cols, k = smp.ref, smp.cols, 64
    target = smp.b.astype(np.float32)
    mats = [lib.ref_csr_new(k, EVAL_BATCH, cols, smp.idx[i * EVAL_BATCH:].ctypes.data_as(C.c_void_p))
            for i in range(nb)]
    w = np.zeros(cols, np.float32)
    m1, m2 = np.zeros_like(w), np.zeros_like(w)
    score, grad = np.empty(EVAL_BATCH, np.float32), np.empty(cols, np.float32)
    b1, b2, eps = 0.9, 0.999, 1e-8
    order = np.random.default_rng(seed).permutation(nb)
    try:
        t0 = time.perf_counter()
        for step, i in enumerate(order, 1):
            lib.ref_csr_mul(mats[i], w.ctypes.data_as(C.c_void_p), score.ctypes.data_as(C.c_void_p))
            d = score - target[i * EVAL_BATCH:(i + 1) * EVAL_BATCH]
            ad = np.abs(d)
            _loss = float(np.mean(np.where(ad <= EVAL_DELTA, 0.5 * d * d, EVAL_DELTA * (ad - 0.5 * EVAL_DELTA)))
                          + EVAL_L2 * np.dot(w, w))
            dsc = (np.clip(d, -EVAL_DELTA, EVAL_DELTA) / EVAL_BATCH).astype(np.float32)
            lib.ref_csr_tmul(mats[i], dsc.ctypes.data_as(C.c_void_p), grad.ctypes.data_as(C.c_void_p))
            grad += (2 * EVAL_L2) * w
            m1 = b1 * m1 + (1 - b1) * grad
            m2 = b2 * m2 + (1 - b2) * grad * grad
            w -= (EVAL_LR / (1 - b1 ** step)) * m1 / (np.sqrt(m2 / (1 - b2 ** step)) + eps)
        per_batch = (time.perf_counter() - t0) / nb
    finally:
        for m in mats:
            lib.ref_csr_free(m)
    return {"value": per_batch * batches_per_epoch, "unit": "s", "cores": _threads(), "kind": "reference",
            "sample": f"{nb} of {batches_per_epoch} minibatches of {EVAL_BATCH} rows (same generator; reference "
                      f"indexing and MatrixCSR built untimed); per minibatch the reference's A*w and g*A plus numpy "
                      f"Huber/Adam, {per_batch * 1e3:.1f} ms; time scaled to the epoch; OpenMP threads "
                      f"{os.environ.get('OMP_NUM_THREADS', os.cpu_count())}"}


def run_reference(args) -> dict | None:
    world, rank, _ = dist_env()
    if rank != 0:
        return None
    import oracle

    if not oracle.ref_available():
        return {"impl": "reference", "metric": METRIC,
                "unavailable": "oracle/_ref (reference sources compiled here) is missing"}
    if args.workload == "evaluator":
        nbatch = -(-args.eval_rows // EVAL_BATCH)
        vals = []
        for i in range(args.warmup + args.steps):
            cbl = cpu_baseline_evaluator(args, args.seed, nbatch)
            if i >= args.warmup:
                vals.append(cbl["value"])
        value = statistics.mean(vals)
        cbl["value"] = value
        return {
            "impl": "reference", "metric": EVAL_METRIC, "value": value, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded random-play positions, seeded targets)", "config": eval_config(args.eval_rows),
            "cpu_baseline": cbl,
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    if args.workload == "batched":
        rows, empties = batched_problems(args.seed, args.problems)
        vals = []
        for i in range(args.warmup + args.steps):
            cbl = cpu_baseline_batched(args, args.seed, rows, empties)
            if i >= args.warmup:
                vals.append(cbl["value"])
        value = statistics.mean(vals)
        cbl["value"] = value
        return {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded random-play positions per empty count, seeded targets)",
            "config": {"workload": f"{args.problems} per-empty-count 8-pattern expanded fits, fitted one after "
                                   f"another with FP64 Jacobi-PCG to {args.tol:g}", "rows": int(rows.sum())},
            "cpu_baseline": cbl,
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    # the single fit: the whole workload every step, on the host cores, with
    # inputs from the oracle's restatement of the seeded generator (the same
    # system the GPU arm builds; this process loads no CUDA library)
    sysm = ReferenceSystem(args.seed, args.rows, args.min_empties, args.max_empties)
    times, last = [], None
    for i in range(args.warmup + args.steps):
        r = sysm.run(args.tol)
        if i >= args.warmup:
            times.append(r["step_s"])
            last = r
    value = statistics.mean(times)
    cbl = {"value": value, "unit": "s", "cores": _threads(), "kind": "reference",
           "sample": f"the whole workload every step ({args.rows} rows): reference indexing "
                     f"({last['index_s']:.2f} s) + FP64 PCG to {args.tol:g} ({last['iterations']} iterations, "
                     f"{last['solve_s']:.2f} s, rel {last['rel_residual']:.2e}); OpenMP threads {_threads()}"}
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded random-play positions, seeded targets)",
        "config": single_config(args), "precision": "FP64 (the reference's Math/ retyped from float)",
        "breakdown": {"index_s": last["index_s"], "solve_s": last["solve_s"], "iterations": last["iterations"],
                      "rel_residual": last["rel_residual"], "steps_s": times},
        "cpu_baseline": cbl,
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main(argv=None) -> int:
    args = parse_args(argv)
    if args.impl == "reference":
        res = run_reference(args)
    elif args.workload == "batched":
        res = run_ours_batched(args)
    elif args.workload == "evaluator":
        res = run_ours_evaluator(args)
    elif dist_env()[0] > 1 or args.sharded:
        res = run_ours_sharded(args)
    else:
        res = run_ours(args)
    if res is not None:
        print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
