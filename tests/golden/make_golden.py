"""Generates the golden fixtures in this directory by running the reference's
own code (compiled from the reference tree by oracle/Makefile into
oracle/_ref/).  Run from the repository root after `make -C oracle ref`:

    python tests/golden/make_golden.py

Outputs (all small, committed):
  indexer_ref.npz  positions of RandomPositionGenerator(1337) (the reference's
                   own fuzz seed, PatternTest/Indexer.cpp:11) and
                   GroupIndexer indices for each fixture pattern
                   (PatternTest/Pattern.h:4-93 restated as masks) and for the
                   5- and 8-pattern fitting sets; CreateIndexer facts.
  math_ref.npz     FP32 reference products on a seeded 200 x 24 CSR, and
                   10 FP32 PCG / LSQR iterations on the 5-pattern system of
                   the fuzz positions with seeded targets.
  flips_ref.npz    the four flips of seeded random bitboards.
  lsmr_ref.npz     10 FP32 LSMR iterations of the reference (Math/Solver.h:
                   222-287) on the 5-pattern system of math_ref.npz.
  estimator_ref.npz  a PatternBasedEstimator file written by the reference's
                   Save (IO/Binary.cpp:46-63) for ESTIMATOR_MASKS with seeded
                   dense weights (stage size 33: 2 stages; 0xFF00 is stored flipped) and the default
                   accuracy model, its file bytes, and the reference's
                   MultiStageScoreEstimator::Eval and Weights() of it on the
                   fuzz positions.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent

# PatternTest/Pattern.h:4-93 as masks (bit 0 = H8; the literal's last character
# is bit 0): a = G8,H8; c = A7,B8; d = H7,G8; h = A8,H8; v = H1,H8;
# vh = B1,G1,B8,G8; dc = B1,A2,H7,G8; vhdc = A1,H1,A8,H8.
FIXTURES = {
    "a": 0x0000000000000003,
    "c": 0x0000000000008040,
    "d": 0x0000000000000102,
    "h": 0x0000000000000081,
    "v": 0x0100000000000001,
    "vh": 0x4200000000000042,
    "dc": 0x4080000000000102,
    "vhdc": 0x8100000000000081,
}
SET5 = [0x42FF, 0x070707, 0x1F1F, 0x8040201008040201, 0xFF00]
# Every indexer class of CreateIndexer, small enough for a committed file.
ESTIMATOR_MASKS = [FIXTURES["a"], FIXTURES["v"], FIXTURES["vh"], FIXTURES["dc"], FIXTURES["vhdc"],
                   FIXTURES["d"], 0x8040201008040201, 0xFF00]
ESTIMATOR_STAGE_SIZE = 33
DEFAULT_ACCURACY = [-0.16594754, 0.95554334, 0.27973529, -0.01616647, 1.28078789]
SET8 = SET5 + [0xFF0000, 0xFF000000, 0x0080402010080402]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def ref_index(masks, pos):
    lib = oracle.ref_lib()
    m = np.asarray(masks, dtype=np.uint64)
    cols = np.zeros(1, np.int64)
    k = lib.ref_group_info(_p(m), len(m), _p(cols), None)
    out = np.empty((len(pos), k), np.uint32)
    lib.ref_group_index(_p(m), len(m), _p(pos), len(pos), _p(out))
    return out, int(cols[0])


def main() -> None:
    lib = oracle.ref_lib()
    n = 2000
    pos = np.empty((n, 2), np.uint64)
    lib.ref_random_positions(1337, n, _p(pos))
    data = {"positions": pos}
    sets = {**{k: [v] for k, v in FIXTURES.items()}, "mix": list(FIXTURES.values()), "set5": SET5, "set8": SET8}
    for name, masks in sets.items():
        idx, cols = ref_index(masks, pos)
        data[f"idx_{name}"] = idx
        data[f"cols_{name}"] = np.int64(cols)
        data[f"masks_{name}"] = np.asarray(masks, np.uint64)
        var = np.empty(idx.shape[1], np.uint64)
        lib.ref_group_info(_p(data[f"masks_{name}"]), len(masks), _p(np.zeros(1, np.int64)), _p(var))
        data[f"variations_{name}"] = var
    info = []
    for m in SET8 + list(FIXTURES.values()):
        sp, order, space = np.zeros(1, np.uint64), np.zeros(1, np.int32), np.zeros(1, np.int32)
        lib.ref_create_indexer(m, _p(sp), _p(order), _p(space))
        info.append((m, int(sp[0]), int(order[0]), int(space[0])))
    data["create_indexer"] = np.array(info, dtype=np.uint64)
    np.savez_compressed(OUT / "indexer_ref.npz", **data)

    rng = np.random.default_rng(20240601)
    rows, k, cols = 200, 24, 150
    idx = rng.integers(0, cols, size=(rows, k)).astype(np.uint32)
    idx[:, 1] = idx[:, 0]  # duplicates within rows
    x = rng.standard_normal(cols).astype(np.float32)
    y = rng.standard_normal(rows).astype(np.float32)
    ax = np.empty(rows, np.float32)
    aty = np.empty(cols, np.float32)
    jac = np.empty(cols, np.float32)
    lib.ref_spmv(k, rows, cols, _p(idx), _p(x), _p(ax))
    lib.ref_spmv_t(k, rows, cols, _p(idx), _p(y), _p(aty))
    lib.ref_jacobi(k, rows, cols, _p(idx), _p(jac))
    # 10 FP32 PCG / LSQR iterations (FitWeights' solve) on a pattern system:
    # the 5-pattern set on the fuzz positions, seeded targets.
    pidx, pcols = ref_index(SET5, pos)
    w = rng.normal(0, 0.5, pcols)
    pb = np.empty(n, np.float64)
    for r in range(n):
        pb[r] = w[pidx[r]].sum()
    pb = np.clip(2 * np.rint((pb + rng.normal(0, 4, n)) / 2), -64, 64).astype(np.float32)
    pk = pidx.shape[1]
    xp = np.empty(pcols, np.float32)
    xl = np.empty(pcols, np.float32)
    rp, rl = C.c_float(), C.c_float()
    lib.ref_pcg(pk, n, pcols, _p(pidx), _p(pb), 10, _p(xp), C.byref(rp))
    lib.ref_lsqr(pk, n, pcols, _p(pidx), _p(pb), 10, _p(xl), C.byref(rl))
    np.savez_compressed(OUT / "math_ref.npz", idx=idx, cols=np.int64(cols), x=x, y=y, ax=ax, aty=aty, jacobi=jac,
                        fit_idx=pidx, fit_cols=np.int64(pcols), fit_b=pb, pcg10_x=xp,
                        pcg10_residuum=np.float32(rp.value), lsqr10_x=xl, lsqr10_residuum=np.float32(rl.value))

    boards = rng.integers(0, 2**63, size=64, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, 64, dtype=np.uint64)
    flips = np.array([[lib.ref_flip(w, int(bb)) for w in range(4)] for bb in boards], dtype=np.uint64)
    np.savez_compressed(OUT / "flips_ref.npz", boards=boards, flips=flips)
    estimator_fixture(lib, pos)
    lsmr_fixture(lib)
    print("wrote", *(p.name for p in OUT.glob("*.npz")))


def estimator_fixture(lib, pos) -> None:
    import os
    import tempfile

    m = np.asarray(ESTIMATOR_MASKS, np.uint64)
    cols = np.zeros(1, np.int64)
    lib.ref_group_info(_p(m), len(m), _p(cols), None)
    c = int(cols[0])
    stages = -(-65 // ESTIMATOR_STAGE_SIZE)
    w = np.random.default_rng(20).normal(0, 2, (stages, c)).astype(np.float32)
    acc = np.asarray(DEFAULT_ACCURACY, np.float32)
    fd, path = tempfile.mkstemp(suffix=".bin")
    os.close(fd)
    try:
        lib.ref_save_estimator(path.encode(), ESTIMATOR_STAGE_SIZE, _p(m), len(m), _p(w), c, _p(acc), len(acc))
        blob = np.frombuffer(Path(path).read_bytes(), np.uint8).copy()
    finally:
        os.unlink(path)
    scores = np.zeros(len(pos), np.float32)
    lib.ref_msse_eval(ESTIMATOR_STAGE_SIZE, _p(m), len(m), _p(w), c, _p(pos), len(pos), _p(scores))
    back = np.zeros_like(w)
    for st in range(stages):
        lib.ref_estimator_weights(_p(m), len(m), _p(w[st]), c, _p(back[st]))
    stored = np.zeros(len(m), np.uint64)
    for i, mk in enumerate(m):
        sp, o, sz = np.zeros(1, np.uint64), np.zeros(1, np.int32), np.zeros(1, np.int32)
        lib.ref_create_indexer(int(mk), _p(sp), _p(o), _p(sz))
        stored[i] = sp[0]
    np.savez_compressed(OUT / "estimator_ref.npz", masks=m, stored=stored, stage_size=np.int32(ESTIMATOR_STAGE_SIZE),
                        weights=w, accuracy=acc, file_bytes=blob, positions=pos, scores=scores, weights_back=back)


if __name__ == "__main__":
    main()


def lsmr_fixture(lib) -> None:
    g = np.load(OUT / "math_ref.npz")
    idx, cols, b = g["fit_idx"], int(g["fit_cols"]), g["fit_b"].astype(np.float32)
    x = np.zeros(cols, np.float32)
    res = C.c_float()
    lib.ref_lsmr(idx.shape[1], idx.shape[0], cols, _p(idx), _p(b), 10, _p(x), C.byref(res))
    np.savez_compressed(OUT / "lsmr_ref.npz", lsmr10_x=x, lsmr10_residuum=np.float32(res.value))
