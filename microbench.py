"""Timing of the two sparse products on one layout, for profiling and tuning.

    python microbench.py --rows 2000000 --layout blocked --reps 3

Builds the 8-pattern expanded matrix of `rows` random-play positions (empty
counts 20..40) on the requested layout, runs A x and A'y `reps` times each
(after two warm-up launches) with CUDA events on the current stream, and
prints one JSON line with seconds and GB/s of algorithmic bytes per product.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
from pathlib import Path

import torch

sys.path.insert(0, str(Path(__file__).resolve().parent))

from cassandra_b200 import PATTERNS_8, GroupIndexer, MatrixCSR, generate_positions  # noqa: E402
from cassandra_b200 import _lib as L  # noqa: E402


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--rows", type=int, default=2_000_000)
    ap.add_argument("--layout", choices=["blocked", "rows"], default="blocked")
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f32")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=7)
    args = ap.parse_args(argv)

    lib = L.load()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    pos = generate_positions(args.seed, args.rows, 20, 40)
    g = GroupIndexer(PATTERNS_8, "expanded")
    a = MatrixCSR.from_positions(g, pos, args.layout)
    del pos
    R, cols, K = a.rows(), a.cols(), a.nnz_per_row
    dt = torch.float32 if args.dtype == "f32" else torch.float64
    code = L.CAS_F32 if args.dtype == "f32" else L.CAS_F64
    es = 4 if args.dtype == "f32" else 8
    x = torch.randn(cols, dtype=dt, device="cuda")
    y = torch.randn(R, dtype=dt, device="cuda")
    yo = torch.empty(R, dtype=dt, device="cuda")
    xo = torch.empty(cols, dtype=dt, device="cuda")

    def timed(fn):
        for _ in range(2):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / args.reps * 1e-3

    t_ax = timed(lambda: L.check(lib.cas_spmv(a.handle, code, C.c_void_p(x.data_ptr()), C.c_void_p(yo.data_ptr()),
                                              sp)))
    t_aty = timed(lambda: L.check(lib.cas_spmv_t(a.handle, code, C.c_void_p(y.data_ptr()),
                                                 C.c_void_p(xo.data_ptr()), sp)))
    nnz = R * K
    idx_ax = (2 if args.layout == "blocked" else 4) * nnz
    idx_aty = 4 * nnz + (0 if args.layout == "blocked" else 8 * (cols + 1))
    bx = idx_ax + es * (R + cols)
    bt = idx_aty + es * (R + cols)
    print(json.dumps({"rows": R, "cols": cols, "nnz": nnz, "layout": args.layout, "dtype": args.dtype,
                      "ax_s": t_ax, "ax_gbs": bx / t_ax / 1e9, "ax_bytes": bx,
                      "aty_s": t_aty, "aty_gbs": bt / t_aty / 1e9, "aty_bytes": bt,
                      "aty_schedules": a.schedules() if args.layout == "blocked" else None}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
