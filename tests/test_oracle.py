"""Pins the C oracle (oracle/oracle.c) to the reference: its golden vectors,
the reference tests' known answers, and the compiled reference itself.
CPU only."""
import ctypes as C

import numpy as np
import pytest

from tests.golden.make_golden import FIXTURES, SET5, SET8


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


# BoardTest/BitBoard.cpp:6-24
@pytest.mark.parametrize("which,expected", [(0, 0x8080808000000000), (1, 0x01010101), (2, 0xF0),
                                            (3, 0x0F00000000000000)])
def test_flip_known_answers(orc, which, expected):
    assert orc.c_lib().or_flip(which, 0xF) == expected


def test_flips_match_golden(orc, golden_flips):
    for b, f in zip(golden_flips["boards"], golden_flips["flips"]):
        assert [orc.c_lib().or_flip(w, int(b)) for w in range(4)] == [int(v) for v in f]


def test_fast_index_matches_reference(orc, ref, golden_indexer):
    pos = golden_indexer["positions"][:300]
    for m in SET8 + list(FIXTURES.values()):
        for p, o in pos:
            assert orc.c_lib().or_fast_index(int(p), int(o), m) == ref.ref_lib().ref_fast_index(int(p), int(o), m)


@pytest.mark.parametrize("name", list(FIXTURES) + ["mix", "set5", "set8"])
def test_group_index_matches_golden(orc, golden_indexer, name):
    masks = golden_indexer[f"masks_{name}"]
    cols, k = orc.group_info(masks, 0)
    assert cols == int(golden_indexer[f"cols_{name}"])
    got = orc.group_index(masks, 0, golden_indexer["positions"])
    np.testing.assert_array_equal(got, golden_indexer[f"idx_{name}"])


def test_group_index_matches_reference_on_random_play(orc, ref):
    import cassandra_b200 as cb

    pos = cb.generate_positions_host(7, 0, 3000, 10, 55)
    for masks in (SET5, SET8, list(FIXTURES.values())):
        m = np.asarray(masks, np.uint64)
        cols = np.zeros(1, np.int64)
        k = ref.ref_lib().ref_group_info(_p(m), len(m), _p(cols), None)
        want = np.empty((len(pos), k), np.uint32)
        ref.ref_lib().ref_group_index(_p(m), len(m), _p(pos), len(pos), _p(want))
        np.testing.assert_array_equal(orc.group_index(m, 0, pos), want)


# PatternTest/Indexer.cpp:8-47: index multisets are invariant under the 8 symmetries
@pytest.mark.parametrize("mode", [0, 1])
def test_symmetry_invariance(orc, golden_indexer, mode):
    pos = golden_indexer["positions"][:500].astype(np.uint64)
    lib = orc.c_lib()

    def flip(w, a):
        return np.array([[lib.or_flip(w, int(p)), lib.or_flip(w, int(o))] for p, o in a], dtype=np.uint64)

    variants = [pos, flip(0, pos), flip(1, pos), flip(2, pos), flip(3, pos), flip(0, flip(2, pos)),
                flip(1, flip(2, pos)), flip(3, flip(2, pos))]
    for masks in ([FIXTURES[k]] for k in FIXTURES):
        if mode == 1 and len(masks) == 1:
            pass
        base = np.sort(orc.group_index(masks, mode, pos), axis=1)
        for v in variants[1:]:
            np.testing.assert_array_equal(np.sort(orc.group_index(masks, mode, v), axis=1), base)
    base = np.sort(orc.group_index(list(FIXTURES.values()), mode, pos), axis=1)
    for v in variants[1:]:
        np.testing.assert_array_equal(np.sort(orc.group_index(list(FIXTURES.values()), mode, v), axis=1), base)


# PatternTest/Indexer.cpp:51-92: all configurations cover the index space
@pytest.mark.parametrize("name", list(FIXTURES))
def test_configurations_cover_index_space(orc, ref, name):
    m = FIXTURES[name]
    n = ref.ref_lib().ref_configurations(m, None)
    conf = np.empty((n, 2), np.uint64)
    ref.ref_lib().ref_configurations(m, _p(conf))
    cols, _ = orc.group_info([m], 0)
    got = np.unique(orc.group_index([m], 0, conf))
    np.testing.assert_array_equal(got, np.arange(cols, dtype=np.uint32))


# MathTest/MatrixCSR.cpp:3-55
def test_matrix_csr_known_answers(orc):
    idx = np.array([[0, 1], [1, 2], [3, 3]], np.uint32)
    np.testing.assert_array_equal(orc.spmv(idx, 4, np.array([1, 2, 3, 4.0])), [3, 5, 8])
    np.testing.assert_array_equal(orc.spmv_t(idx, 4, np.array([1, 2, 3.0])), [1, 3, 2, 6])
    np.testing.assert_array_equal(orc.jacobi(idx, 4), [1, 0.5, 1, 0.25])


def test_products_match_reference_fp32_golden(orc, golden_math):
    g = golden_math
    cols = int(g["cols"])
    np.testing.assert_allclose(orc.spmv(g["idx"], cols, g["x"].astype(np.float64)), g["ax"], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(orc.spmv_t(g["idx"], cols, g["y"].astype(np.float64)), g["aty"], rtol=1e-5,
                               atol=1e-5)
    np.testing.assert_allclose(orc.jacobi(g["idx"], cols), g["jacobi"], rtol=1e-6)


def test_products_match_reference_fp64(orc, ref):
    rng = np.random.default_rng(3)
    rows, k, cols = 3000, 40, 997
    idx = rng.integers(0, cols, size=(rows, k)).astype(np.uint32)
    idx[:, 5] = idx[:, 4]
    x = rng.standard_normal(cols)
    y = rng.standard_normal(rows)
    lib = ref.ref64_lib()
    want = np.empty(rows)
    lib.ref64_spmv(k, rows, cols, _p(idx), _p(x), _p(want))
    np.testing.assert_allclose(orc.spmv(idx, cols, x), want, rtol=1e-13)
    want = np.empty(cols)
    lib.ref64_spmv_t(k, rows, cols, _p(idx), _p(y), _p(want))
    np.testing.assert_allclose(orc.spmv_t(idx, cols, y), want, rtol=1e-11, atol=1e-11)
    want = np.empty(cols)
    with np.errstate(divide="ignore"):
        lib.ref64_jacobi(k, rows, cols, _p(idx), _p(want))
    np.testing.assert_array_equal(orc.jacobi(idx, cols), want)


def test_kept_matrix_products_match_reference_calls(ref):
    """The reference's products on a MatrixCSR kept across calls (the
    evaluator's CPU baseline) equal the same products on a matrix built for
    each call; with integer-valued vectors every FP32 sum is exact."""
    lib = ref.ref_lib()
    rng = np.random.default_rng(5)
    rows, k, cols = 2000, 16, 501
    idx = rng.integers(0, cols, size=(rows, k)).astype(np.uint32)
    x = rng.integers(-8, 9, cols).astype(np.float32)
    y = rng.integers(-8, 9, rows).astype(np.float32)
    m = lib.ref_csr_new(k, rows, cols, _p(idx))
    try:
        got, want = np.empty(rows, np.float32), np.empty(rows, np.float32)
        lib.ref_csr_mul(m, _p(x), _p(got))
        lib.ref_spmv(k, rows, cols, _p(idx), _p(x), _p(want))
        np.testing.assert_array_equal(got, want)
        np.testing.assert_array_equal(got, x[idx].sum(axis=1))
        got, want = np.empty(cols, np.float32), np.empty(cols, np.float32)
        lib.ref_csr_tmul(m, _p(y), _p(got))
        lib.ref_spmv_t(k, rows, cols, _p(idx), _p(y), _p(want))
        np.testing.assert_array_equal(got, want)
        exact = np.zeros(cols)
        np.add.at(exact, idx.ravel(), np.repeat(y.astype(np.float64), k))
        np.testing.assert_array_equal(got, exact.astype(np.float32))
    finally:
        lib.ref_csr_free(m)


def _small_system(orc, rows=4000, seed=11):
    import cassandra_b200 as cb

    pos = cb.generate_positions_host(seed, 0, rows, 20, 40)
    idx = orc.group_index(SET5, 0, pos)
    cols, _ = orc.group_info(SET5, 0)
    rng = np.random.default_rng(seed)
    w = rng.normal(0, 0.5, cols)
    b = np.clip(2 * np.rint((orc.spmv(idx, cols, w) + rng.normal(0, 4, rows)) / 2), -64, 64)
    return idx, cols, b


def _ref64_pcg(ref, idx, cols, b, iters):
    want = np.empty(cols)
    rel, sec = np.zeros(1), np.zeros(1)
    n = ref.ref64_lib().ref64_pcg(idx.shape[1], idx.shape[0], cols, _p(idx), _p(np.ascontiguousarray(b, np.float64)),
                                  iters, 0.0, iters, _p(want), _p(rel), _p(sec))
    assert n == iters
    return want, rel[0]


def test_pcg_matches_reference_fp64(orc, ref):
    """Same iterates as the reference's PCG retyped to FP64 (run on one
    thread: with more, its sums merge in arrival order and the target moves
    run to run).  CG amplifies the rounding of differently ordered sums, so
    iterates agree to ~1e-14 after 10 steps and, after 60, the residuals and
    predictions agree to the stated looser bounds."""
    idx, cols, b = _small_system(orc)
    x, res, it = orc.pcg(idx, cols, b, 10)
    assert it == 10
    with orc.single_thread():
        want, _ = _ref64_pcg(ref, idx, cols, b, 10)
    np.testing.assert_allclose(x, want, rtol=0, atol=1e-11 * np.abs(want).max())
    x, res, it = orc.pcg(idx, cols, b, 60)
    with orc.single_thread():
        want, rel = _ref64_pcg(ref, idx, cols, b, 60)
    assert abs(orc.normal_residual(idx, cols, b, x) - rel) <= 1e-2 * rel
    aw = orc.spmv(idx, cols, want)
    np.testing.assert_allclose(orc.spmv(idx, cols, x), aw, rtol=0, atol=1e-5 * np.abs(aw).max())


def test_pcg_matches_reference_fp32_golden(orc, golden_math):
    g = golden_math
    x, res, _ = orc.pcg(g["fit_idx"], int(g["fit_cols"]), g["fit_b"].astype(np.float64), 10)
    np.testing.assert_allclose(x, g["pcg10_x"], rtol=0, atol=1e-4 * np.abs(g["pcg10_x"]).max())
    np.testing.assert_allclose(res, g["pcg10_residuum"], rtol=2e-3)


def _ref64_lsqr(ref, idx, cols, b, iters):
    want = np.empty(cols)
    rel, sec = np.zeros(1), np.zeros(1)
    ref.ref64_lib().ref64_lsqr(idx.shape[1], idx.shape[0], cols, _p(idx), _p(np.ascontiguousarray(b, np.float64)),
                               iters, 0.0, iters, _p(want), _p(rel), _p(sec))
    return want, rel[0]


def test_lsqr_matches_reference(orc, ref, golden_math):
    """Unpreconditioned LSQR on these rank-deficient systems amplifies a 1e-15
    perturbation of b to ~1e-7 in 10 steps (measured), so iterates are pinned
    tightly after 5 steps and through ||b - Ax|| after 40."""
    idx, cols, b = _small_system(orc, rows=3000, seed=5)
    x, res, it = orc.lsqr(idx, cols, b, 5)
    want, _ = _ref64_lsqr(ref, idx, cols, b, 5)
    np.testing.assert_allclose(x, want, rtol=0, atol=1e-9 * np.abs(want).max())
    x, res, it = orc.lsqr(idx, cols, b, 40)
    want, rel = _ref64_lsqr(ref, idx, cols, b, 40)
    # The reference's own FP64 LSQR is not reproducible run to run at 40 steps
    # (its x * A merges thread-private sums in arrival order; measured ||b-Ax||
    # 7.068 / 7.088 / 7.093 in three runs), so the oracle is held to that spread
    # and to its own consistency: phi_bar equals ||b - Ax||.
    r_got = np.linalg.norm(b - orc.spmv(idx, cols, x))
    r_want = np.linalg.norm(b - orc.spmv(idx, cols, want))
    assert abs(r_got - r_want) <= 2e-2 * r_want
    assert abs(res - r_got) <= 1e-9 * r_got
    g = golden_math
    x, res, _ = orc.lsqr(g["fit_idx"], int(g["fit_cols"]), g["fit_b"].astype(np.float64), 10)
    np.testing.assert_allclose(x, g["lsqr10_x"], rtol=0, atol=1e-3 * np.abs(g["lsqr10_x"]).max())
    np.testing.assert_allclose(res, g["lsqr10_residuum"], rtol=2e-3)


def _ref64_lsmr(ref, idx, cols, b, iters):
    want = np.empty(cols)
    rel, sec = np.zeros(1), np.zeros(1)
    with ref.single_thread():
        ref.ref64_lib().ref64_lsmr(idx.shape[1], idx.shape[0], cols, _p(idx),
                                   _p(np.ascontiguousarray(b, np.float64)), iters, 0.0, iters, _p(want), _p(rel),
                                   _p(sec))
    return want, rel[0]


def test_lsmr_matches_reference(orc, ref):
    """The oracle's LSMR (Math/Solver.h:222-287 with its Givens rotations)
    against the reference's own LSMR retyped to FP64, single-threaded:
    iterates agree to rounding after 5 and 40 steps."""
    idx, cols, b = _small_system(orc, rows=3000, seed=5)
    for steps in (5, 40):
        x, zeta_bar, it = orc.lsmr(idx, cols, b, steps)
        want, rel = _ref64_lsmr(ref, idx, cols, b, steps)
        assert it == steps
        np.testing.assert_allclose(x, want, rtol=0, atol=1e-12 * np.abs(want).max())
        assert abs(orc.normal_residual(idx, cols, b, x) - rel) <= 1e-9 * rel


def test_lsmr_golden(orc):
    """10 FP32 steps of the reference's LSMR (committed fixture) against the
    FP64 oracle on the 5-pattern system: FP32 rounding only."""
    g = np.load("tests/golden/math_ref.npz")
    lg = np.load("tests/golden/lsmr_ref.npz")
    x, _, _ = orc.lsmr(g["fit_idx"], int(g["fit_cols"]), g["fit_b"].astype(np.float64), 10)
    np.testing.assert_allclose(x, lg["lsmr10_x"], rtol=0, atol=1e-3 * np.abs(lg["lsmr10_x"]).max())
    assert float(lg["lsmr10_residuum"]) == 0.0  # LSMR::Residuum() returns 0 (Math/Solver.h:284)


def test_lsmr_reaches_tolerance(orc):
    idx, cols, b = _small_system(orc, rows=3000, seed=2)
    x, _, it = orc.lsmr(idx, cols, b, 20000, tol=1e-8, check_every=10)
    assert orc.normal_residual(idx, cols, b, x) <= 1e-8 and it < 20000


def test_pcg_reaches_tolerance(orc):
    idx, cols, b = _small_system(orc, rows=3000, seed=2)
    x, res, it = orc.pcg(idx, cols, b, 5000, tol=1e-8, check_every=10)
    assert it < 5000
    assert orc.normal_residual(idx, cols, b, x) <= 1e-8


def _scaled_matrix(orc, idx, cols):
    """A S as a scipy matrix, S = diag(A'A)^-1/2 (1 for an empty column)."""
    import scipy.sparse as sp

    d = orc.jacobi(idx, cols)
    s = np.where(np.isfinite(d) & (d > 0), np.sqrt(np.where(np.isfinite(d), d, 1.0)), 1.0)
    rows, k = idx.shape
    a = sp.csr_matrix((np.ones(idx.size), idx.ravel().astype(np.int64), np.arange(0, idx.size + 1, k)),
                      shape=(rows, cols))
    return a @ sp.diags(s), s


@pytest.mark.parametrize("method", ["lsqr", "lsmr"])
def test_scaled_least_squares_match_scipy(orc, method):
    """The column-scaled LSQR/LSMR of the oracle (not in the reference) are
    the published methods on A S: after 10 steps x = S y equals scipy's
    lsqr/lsmr on the explicit matrix A S with no stopping test (scipy's
    LSMR is the Fong-Saunders method whose rotations Math/Solver.h:222-287
    follow)."""
    import scipy.sparse.linalg as sla

    idx, cols, b = _small_system(orc, rows=3000, seed=5)
    a_s, s = _scaled_matrix(orc, idx, cols)
    fn = orc.lsqr if method == "lsqr" else orc.lsmr
    x, _, it = fn(idx, cols, b, 10, scale=True)
    assert it == 10
    solver = sla.lsqr if method == "lsqr" else sla.lsmr
    y = solver(a_s, b, atol=0, btol=0, conlim=0, maxiter=10)[0] if method == "lsmr" else \
        sla.lsqr(a_s, b, atol=0, btol=0, conlim=0, iter_lim=10)[0]
    np.testing.assert_allclose(x, s * y, rtol=0, atol=1e-9 * np.abs(x).max())


@pytest.mark.parametrize("method", ["lsqr", "lsmr"])
def test_scaled_least_squares_reach_tolerance(orc, method):
    """Column scaling leaves the least-squares problem unchanged: the scaled
    solves reach 1e-8 on the normal equations, in fewer steps than the
    unscaled ones (140 against 290 LSQR steps here), with the predictions
    A x of the PCG solution."""
    idx, cols, b = _small_system(orc, rows=3000, seed=2)
    fn = orc.lsqr if method == "lsqr" else orc.lsmr
    x, _, it = fn(idx, cols, b, 20000, tol=1e-8, check_every=10, scale=True)
    assert orc.normal_residual(idx, cols, b, x) <= 1e-8
    _, _, it_plain = fn(idx, cols, b, 20000, tol=1e-8, check_every=10)
    assert it < it_plain
    xp, _, _ = orc.pcg(idx, cols, b, 5000, tol=1e-10, check_every=10)
    pa, pp = orc.spmv(idx, cols, x), orc.spmv(idx, cols, xp)
    assert np.abs(pa - pp).max() <= 1e-5 * np.abs(pp).max()


@pytest.mark.parametrize("seed,first,n,lo,hi", [(2024, 0, 20_000, 20, 40), (7, 123_456, 5000, 0, 60),
                                                (1, 0, 3000, 60, 60), (99, 10 ** 9, 2000, 1, 1)])
def test_generator_restatement_equals_library(orc, seed, first, n, lo, hi):
    """The oracle's C restatement of the seeded random-play generator (used
    where the CUDA library must not be loaded) gives the library's host
    generator's positions bit for bit."""
    import cassandra_b200 as cb

    want = cb.generate_positions_host(seed, first, n, lo, hi).reshape(-1, 2).view(np.uint64)
    np.testing.assert_array_equal(orc.generate_positions(seed, first, n, lo, hi), want)


def test_generated_targets_follow_their_recipe(orc):
    """b = clamp(2 rint((A w* + e) / 2), -64, 64): even integers in [-64, 64],
    correlated with A w*, and w* has the requested spread."""
    pos = orc.generate_positions(5, 0, 20_000, 20, 40)
    idx = orc.group_index(SET8, 1, pos)
    cols, _ = orc.group_info(SET8, 1)
    b, w = orc.generate_targets(idx, cols, 5)
    assert np.all(b == 2 * np.rint(b / 2)) and b.min() >= -64 and b.max() <= 64
    assert abs(w.std() - 0.5) < 0.01 and abs(w.mean()) < 0.01
    aw = orc.spmv(idx, cols, w)
    assert np.corrcoef(aw, b)[0, 1] > 0.5
    assert abs(np.std(b - aw) - 4.0) < 0.2
