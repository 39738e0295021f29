"""The blocked layout (16-bit pattern-local columns per 16384-row block and a
per-block column-sorted copy): products and solvers against the oracle and
against the rows layout, on block-boundary sizes and both index modes."""
import numpy as np
import pytest
import torch

import cassandra_b200 as cb
from tests.golden.make_golden import FIXTURES, SET5, SET8

pytestmark = pytest.mark.gpu

ROWS = [1, 7, 16383, 16384, 16385, 50_001]


def _build(rows, masks, mode, layouts, seed=3):
    pos = cb.generate_positions(seed, rows, 10, 50)
    g = cb.GroupIndexer(masks, mode)
    return cb.MatrixCSR.from_positions(g, pos, layouts), pos, g


@pytest.mark.parametrize("rows", ROWS)
@pytest.mark.parametrize("masks,mode", [(SET8, "expanded"), (SET5, "reference"), (list(FIXTURES.values()), "reference")])
def test_blocked_products_match_oracle(cuda, orc, rows, masks, mode):
    a, pos, g = _build(rows, masks, mode, "blocked")
    assert a.layouts() == {"blocked"}
    cols = g.index_space_size
    idx = orc.group_index(masks, 0 if mode == "reference" else 1, pos.cpu().numpy().view(np.uint64))
    rng = np.random.default_rng(rows)
    x = rng.standard_normal(cols)
    y = rng.standard_normal(rows)
    np.testing.assert_allclose((a @ torch.from_numpy(x).cuda()).cpu().numpy(), orc.spmv(idx, cols, x), rtol=1e-12,
                               atol=1e-11)
    np.testing.assert_allclose((torch.from_numpy(y).cuda() @ a).cpu().numpy(), orc.spmv_t(idx, cols, y), rtol=1e-11,
                               atol=1e-10)
    # FP32: exact for integer-valued vectors
    xi = rng.integers(-50, 50, cols).astype(np.float32)
    yi = rng.integers(-50, 50, rows).astype(np.float32)
    np.testing.assert_array_equal((a @ torch.from_numpy(xi).cuda()).cpu().numpy(),
                                  orc.spmv(idx, cols, xi.astype(np.float64)).astype(np.float32))
    np.testing.assert_array_equal((torch.from_numpy(yi).cuda() @ a).cpu().numpy(),
                                  orc.spmv_t(idx, cols, yi.astype(np.float64)).astype(np.float32))
    # FP32, general values: within FP32 accumulation error
    x32 = x.astype(np.float32)
    got = (a @ torch.from_numpy(x32).cuda()).cpu().numpy().astype(np.float64)
    want = orc.spmv(idx, cols, x32.astype(np.float64))
    assert np.abs(got - want).max() <= 64 * 2 ** -23 * np.abs(want).max() + 1e-6
    with np.errstate(divide="ignore"):
        np.testing.assert_array_equal(cb.jacobi_preconditioner_of_ata(a).cpu().numpy(), orc.jacobi(idx, cols))


SCHEDULES = ["4,0,2,0,0", "4,0,1,1,0", "3,0,2,1,1", "2,0,2,0,1", "2,1,2,1,0", "1,1,2,0,0", "2,1,3,1,1",
             "4,1,6,0,1", "1,0,5,1,1"]


@pytest.mark.parametrize("sched", SCHEDULES)
def test_aty_schedules_match_oracle(cuda, orc, monkeypatch, sched):
    """Every A'y schedule the autotuner can pick (forced through
    CAS_ATY_SCHEDULE): exact on integer-valued FP32 vectors, on a matrix with
    a partial last block and heavy columns (narrow empty-count range)."""
    monkeypatch.setenv("CAS_ATY_SCHEDULE", sched)
    rows = 3 * 16384 + 1234
    a, pos, g = _build(rows, SET8, "expanded", "blocked", seed=31)
    want = tuple(int(v) for v in sched.split(","))
    cur = a.schedules()["in_use"]
    assert (cur["chunks_per_item"], cur["range_major"], cur["items_per_sm"], cur["pack"], cur["persistent"]) == want
    idx = orc.group_index(SET8, 1, pos.cpu().numpy().view(np.uint64))
    yi = np.random.default_rng(5).integers(-50, 50, rows).astype(np.float32)
    np.testing.assert_array_equal((torch.from_numpy(yi).cuda() @ a).cpu().numpy(),
                                  orc.spmv_t(idx, g.index_space_size, yi.astype(np.float64)).astype(np.float32))
    y = torch.randn(rows, dtype=torch.float32, device="cuda")
    assert (y @ a).cpu().numpy().tobytes() == (y @ a).cpu().numpy().tobytes()  # persistent CTAs: same bits
    # the Jacobi diagonal is counted through this schedule's FP32 A'y
    with np.errstate(divide="ignore"):
        np.testing.assert_array_equal(cb.jacobi_preconditioner_of_ata(a).cpu().numpy(),
                                      orc.jacobi(idx, g.index_space_size))


@pytest.mark.parametrize("direct", ["0", "1"])
@pytest.mark.parametrize("rows,masks,mode", [(70_001, SET8, "expanded"), (16385, list(FIXTURES.values()), "reference"),
                                             (300, SET5, "reference")])
def test_jacobi_diagonal_both_paths(cuda, orc, monkeypatch, direct, rows, masks, mode):
    """diag(A'A) from the column counts A'1 plus the repeats' share, and
    counted directly from G32 (the path of layouts whose A'y items are too
    long for exact FP32 counts, forced by CAS_DIAG_FROM_G32=1): both equal
    the oracle's, rows holding a column several times included."""
    monkeypatch.setenv("CAS_DIAG_FROM_G32", direct)
    a, pos, g = _build(rows, masks, mode, "blocked", seed=41)
    idx = orc.group_index(masks, 0 if mode == "reference" else 1, pos.cpu().numpy().view(np.uint64))
    srt = np.sort(idx.astype(np.int64), axis=1)
    assert (srt[:, 1:] == srt[:, :-1]).any()  # repeats present
    with np.errstate(divide="ignore"):
        np.testing.assert_array_equal(cb.jacobi_preconditioner_of_ata(a).cpu().numpy(),
                                      orc.jacobi(idx, g.index_space_size))


def test_autotuner_times_candidates_and_caches(cuda, monkeypatch):
    monkeypatch.delenv("CAS_ATY_SCHEDULE", raising=False)
    rows = 64 * 16384  # smallest layout that is tuned
    a, pos, g = _build(rows, SET8, "expanded", "blocked", seed=32)
    sch = a.schedules()
    timed = sch["timed"]
    assert len(timed) == 12 and all(t["ms"] > 0 for t in timed)
    best = min(timed, key=lambda t: t["ms"])
    cur = sch["in_use"]
    keys = ("chunks_per_item", "range_major", "items_per_sm", "pack", "persistent")
    assert tuple(cur[k] for k in keys) == tuple(best[k] for k in keys)
    b = cb.MatrixCSR.from_positions(g, pos, "blocked")  # same shape: cached, not re-timed
    sb = b.schedules()
    assert sb["timed"] == [] and sb["in_use"]["chunks_per_item"] == cur["chunks_per_item"]


def test_blocked_and_rows_layouts_agree(cuda):
    both, pos, g = _build(40_000, SET8, "expanded", "rows+blocked")
    rows_only = cb.MatrixCSR.from_positions(g, pos, "rows")
    assert both.layouts() == {"rows", "blocked"}
    np.testing.assert_array_equal(both.indices().cpu().numpy(), rows_only.indices().cpu().numpy())
    y = torch.randn(40_000, dtype=torch.float64, device="cuda")
    np.testing.assert_allclose((y @ both).cpu().numpy(), (y @ rows_only).cpu().numpy(), rtol=1e-11, atol=1e-10)
    np.testing.assert_array_equal(cb.jacobi_preconditioner_of_ata(both).cpu().numpy(),
                                  cb.jacobi_preconditioner_of_ata(rows_only).cpu().numpy())


def test_blocked_transpose_is_deterministic(cuda):
    a, pos, g = _build(120_000, SET8, "expanded", "blocked")
    for dt in (torch.float32, torch.float64):
        y = torch.randn(120_000, dtype=dt, device="cuda")
        r1 = (y @ a).cpu().numpy()
        r2 = (y @ a).cpu().numpy()
        assert r1.tobytes() == r2.tobytes()


def test_blocked_rejects_wide_patterns(cuda):
    pos = cb.generate_positions(1, 100, 10, 50)
    g = cb.GroupIndexer([0xFFF], "expanded")  # 12 squares: 531441 columns > 65536
    with pytest.raises(cb.CasError):
        cb.MatrixCSR.from_positions(g, pos, "blocked")
    a = cb.MatrixCSR.from_positions(g, pos)  # default falls back to the rows layout
    assert a.layouts() == {"rows"}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("method", ["pcg", "lsqr"])
def test_solvers_on_blocked_layout(cuda, orc, precision, method):
    rows = 3000 if method == "lsqr" else 40_000
    a, pos, g = _build(rows, SET5 if method == "lsqr" else SET8, "reference" if method == "lsqr" else "expanded",
                       "blocked", seed=9)
    b = cb.generate_targets(a, 9)
    masks = SET5 if method == "lsqr" else SET8
    idx = orc.group_index(masks, 0 if method == "lsqr" else 1, pos.cpu().numpy().view(np.uint64))
    cols = g.index_space_size
    cls = cb.PCG if method == "pcg" else cb.LSQR
    tol = 1e-8
    s = cls(a, b, precision=precision, tol=tol, max_iterations=60_000, check_every=50)
    rep = s.run()
    assert rep["converged"], rep
    assert orc.normal_residual(idx, cols, b.cpu().numpy(), s.x().cpu().numpy()) <= 1.5 * tol


def test_pcg_iterates_on_blocked_match_oracle(cuda, orc):
    a, pos, g = _build(30_000, SET8, "expanded", "blocked", seed=4)
    b = cb.generate_targets(a, 4)
    idx = orc.group_index(SET8, 1, pos.cpu().numpy().view(np.uint64))
    s = cb.PCG(a, b, check_every=5)  # plain FP64 on the blocked layout
    s.iterate(10)
    want, res, _ = orc.pcg(idx, g.index_space_size, b.cpu().numpy(), 10)
    np.testing.assert_allclose(s.x().cpu().numpy(), want, rtol=0, atol=1e-10 * np.abs(want).max())


def test_mixed_solution_matches_plain(cuda):
    """Mixed precision on the blocked layout and plain FP64 on the rows layout
    reach the same least-squares fit (same predictions) at 1e-8."""
    pos = cb.generate_positions(12, 60_000, 20, 40)
    g = cb.GroupIndexer(SET8, "expanded")
    fast = cb.MatrixCSR.from_positions(g, pos, "blocked")
    plain = cb.MatrixCSR.from_positions(g, pos, "rows")
    b = cb.generate_targets(plain, 12)
    m = cb.PCG(fast, b, precision="mixed", tol=1e-8)
    p = cb.PCG(plain, b, precision="fp64", tol=1e-8)
    rm, rp = m.run(), p.run()
    assert rm["converged"] and rp["converged"]
    pm = (plain @ m.x()).cpu().numpy()
    pp = (plain @ p.x()).cpu().numpy()
    np.testing.assert_allclose(pm, pp, rtol=0, atol=1e-5 * np.abs(pp).max())


def test_products_on_a_layout_of_one_unit_per_block(cuda):
    """A layout of more blocks than SMs runs A x with one unit per 16384-row
    block (16 rows per thread) and A'y on its range-major work list: both
    products against the same products on the rows layout, FP32 and FP64,
    over every row and column."""
    rows = 160 * 16384 + 4321
    pos = cb.generate_positions(91, rows, 20, 40)
    g = cb.GroupIndexer(SET8, "expanded")
    fast = cb.MatrixCSR.from_positions(g, pos, "blocked")
    plain = cb.MatrixCSR.from_positions(g, pos, "rows")
    gen = torch.Generator("cuda").manual_seed(3)
    x = torch.randint(-40, 40, (g.index_space_size,), device="cuda", generator=gen).double()
    y = torch.randint(-40, 40, (rows,), device="cuda", generator=gen).double()
    for dt in (torch.float32, torch.float64):
        assert torch.equal((fast @ x.to(dt)).double(), (plain @ x).double())  # integer values: exact
        assert torch.equal((y.to(dt) @ fast).double(), (y @ plain).double())
