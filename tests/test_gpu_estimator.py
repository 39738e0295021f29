"""Pattern-based score estimators on the device (Pattern/Evaluator.cpp):
expansion of dense weights into per-variation tables, batch Eval of a
MultiStageScoreEstimator (bitwise the reference's FP32 sums) and Weights().
Checked against the reference's own outputs (committed fixture), the oracle's
group indices, and the compiled reference where it is available."""
import ctypes as C

import numpy as np
import pytest
import torch

import cassandra_b200 as cb
import oracle

pytestmark = pytest.mark.gpu

GOLD = np.load("tests/golden/estimator_ref.npz")


def _gold_estimator():
    return cb.MultiStageScoreEstimator([int(v) for v in GOLD["masks"]], int(GOLD["stage_size"]), GOLD["weights"])


def test_eval_matches_reference_fixture(cuda):
    e = _gold_estimator()
    pos = torch.from_numpy(GOLD["positions"].view(np.int64)).cuda()
    got = e.eval(pos).cpu().numpy()
    np.testing.assert_array_equal(got.view(np.uint32), GOLD["scores"].view(np.uint32))  # bitwise


def test_weights_and_patterns_match_reference_fixture(cuda):
    e = _gold_estimator()
    assert e.pattern() == [int(v) for v in GOLD["stored"]]
    for st in range(e.stages):
        np.testing.assert_array_equal(e.weights(st).cpu().numpy(), GOLD["weights_back"][st])


def test_tables_follow_the_expansion_rule(cuda, orc):
    """table_i[FastIndex(c, variation_i)] = dense[Indices(c)[i]] for every
    configuration c of variation i (Pattern/Evaluator.cpp:20-26), with the
    oracle's reference-mode group indices as Indices."""
    masks = [int(v) for v in GOLD["masks"]]
    e = _gold_estimator()
    g = cb.GroupIndexer(masks, "reference")
    variations = g.variations()
    tables = e.tables(1).cpu().numpy()
    dense = GOLD["weights"][1]
    off = 0
    for s, var in enumerate(int(v) for v in variations):
        sq = [b for b in range(64) if (var >> b) & 1]
        n = 3 ** len(sq)
        cfg = np.zeros((n, 2), np.uint64)
        for e_ in range(n):
            x, p, o = e_, 0, 0
            for b in sq:
                d = x % 3
                x //= 3
                if d == 1:
                    p |= 1 << b
                elif d == 2:
                    o |= 1 << b
            cfg[e_] = (p, o)
        idx = orc.group_index(masks, 0, cfg)
        np.testing.assert_array_equal(tables[off:off + n], dense[idx[:, s]])
        off += n
    assert off == e.table_floats


def test_file_to_device_estimator(cuda, tmp_path):
    p = tmp_path / "ref.bin"
    p.write_bytes(GOLD["file_bytes"].tobytes())
    e = cb.MultiStageScoreEstimator.load(p)
    pos = torch.from_numpy(GOLD["positions"].view(np.int64)).cuda()
    np.testing.assert_array_equal(e.eval(pos).cpu().numpy().view(np.uint32), GOLD["scores"].view(np.uint32))
    q = tmp_path / "again.bin"
    e.save(q, GOLD["accuracy"])
    assert q.read_bytes() == p.read_bytes()


def test_bad_arguments(cuda):
    masks = [int(v) for v in GOLD["masks"]]
    with pytest.raises(cb.SizeMismatch):
        cb.MultiStageScoreEstimator(masks, 33, GOLD["weights"][:, :-1])
    e = _gold_estimator()
    with pytest.raises(cb.CasError):
        e.tables(e.stages)
    assert e.eval(torch.empty((0, 2), dtype=torch.int64, device="cuda")).numel() == 0


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not compiled here")
@pytest.mark.parametrize("name,stage_size", [("P5", 1), ("P5", 13), ("SET8", 10)])
def test_fitting_sets_match_reference(cuda, name, stage_size):
    """The fitting pattern sets, seeded dense weights per stage, random
    positions of every empty count: scores bitwise the reference's
    MultiStageScoreEstimator::Eval."""
    from tests.golden.make_golden import SET8

    masks = cb.PATTERNS_5 if name == "P5" else SET8
    lib = oracle.ref_lib()
    m = np.asarray(masks, np.uint64)
    cols = cb.GroupIndexer(masks, "reference").index_space_size
    stages = cb.estimator_stages(stage_size)
    w = np.random.default_rng(stage_size).normal(0, 2, (stages, cols)).astype(np.float32)
    n = 20000
    pos = np.empty((n, 2), np.uint64)
    lib.ref_random_positions(77, n, pos.ctypes.data_as(C.c_void_p))
    want = np.empty(n, np.float32)
    lib.ref_msse_eval(stage_size, m.ctypes.data_as(C.c_void_p), len(m), w.ctypes.data_as(C.c_void_p), cols,
                      pos.ctypes.data_as(C.c_void_p), n, want.ctypes.data_as(C.c_void_p))
    e = cb.MultiStageScoreEstimator(masks, stage_size, w)
    got = e.eval(torch.from_numpy(pos.view(np.int64)).cuda()).cpu().numpy()
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("name", ["a", "c", "d", "h", "v", "vh", "dc", "vhdc"])
def test_symmetry_independent_estimator(cuda, orc, name):
    """PatternTest/Evaluator.cpp:7-31 for every fixture pattern: weights
    1..N (N = the pattern's configuration count) survive Weights(), and the
    score of every configuration equals the scores of its 8 symmetric
    variants."""
    from tests.golden.make_golden import FIXTURES

    mask = FIXTURES[name]
    cols = cb.GroupIndexer([mask], "reference").index_space_size
    w = np.arange(1, cols + 1, dtype=np.float32)[None, :]
    e = cb.MultiStageScoreEstimator([mask], 65, w)  # one stage
    np.testing.assert_array_equal(e.weights(0).cpu().numpy(), w[0])
    sq = [b for b in range(64) if (mask >> b) & 1]
    cfg = []
    for code in range(3 ** len(sq)):
        p = o = 0
        for b in sq:
            d = code % 3
            code //= 3
            if d == 1:
                p |= 1 << b
            elif d == 2:
                o |= 1 << b
        cfg.append((p, o))
    cfg = np.array(cfg, np.uint64)
    lib = orc.c_lib()

    def flip(wh, a):
        return np.array([[lib.or_flip(wh, int(p)), lib.or_flip(wh, int(o))] for p, o in a], dtype=np.uint64)

    variants = [cfg, flip(0, cfg), flip(1, cfg), flip(2, cfg), flip(3, cfg), flip(0, flip(2, cfg)),
                flip(1, flip(2, cfg)), flip(3, flip(2, cfg))]
    scores = [e.eval(torch.from_numpy(v.view(np.int64)).cuda()).cpu().numpy() for v in variants]
    for s in scores[1:]:
        np.testing.assert_array_equal(s, scores[0])
