"""Batched per-stage fits (one problem per empty count, as the reference's
training loop fits them one after another, PatternFit/PatternFit.cpp:53-84):
the block-diagonal batch layout and the batched PCG, checked per problem
against the oracle and against single fits."""
import numpy as np
import pytest
import torch

import cassandra_b200 as cb
from tests.golden.make_golden import SET8

pytestmark = pytest.mark.gpu


def _batch(sizes, seed=40, empties=None):
    parts = []
    for q, n in enumerate(sizes):
        e = empties[q] if empties else 12 + (7 * q) % 40
        if n:
            parts.append(cb.generate_positions(seed + q, n, e, e))
    pos = torch.cat(parts) if parts else torch.empty((0, 2), dtype=torch.int64, device="cuda")
    g = cb.GroupIndexer(SET8, "expanded")
    a = cb.MatrixCSR.from_positions_batched(g, pos, sizes)
    return a, pos, g


def _oracle_problems(orc, a, pos):
    row0 = a.problems()
    ph = pos.cpu().numpy().view(np.uint64)
    return row0, [orc.group_index(SET8, 1, ph[row0[q]:row0[q + 1]]) for q in range(len(row0) - 1)]


def test_batched_layout_geometry(cuda):
    sizes = [16385, 1, 0, 7000, 16384]
    a, pos, g = _batch(sizes)
    C = g.index_space_size
    assert a.layouts() == {"blocked"}
    assert a.rows() == sum(sizes) and a.cols() == len(sizes) * C
    np.testing.assert_array_equal(a.problems(), np.concatenate([[0], np.cumsum(sizes)]))


def test_batched_products_match_oracle_per_problem(cuda, orc):
    sizes = [16385, 1, 0, 7000, 16384]
    a, pos, g = _batch(sizes)
    C = g.index_space_size
    row0, idx = _oracle_problems(orc, a, pos)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(a.cols())
    y = rng.standard_normal(a.rows())
    ax = (a @ torch.from_numpy(x).cuda()).cpu().numpy()
    aty = (torch.from_numpy(y).cuda() @ a).cpu().numpy()
    with np.errstate(divide="ignore"):
        jac = cb.jacobi_preconditioner_of_ata(a).cpu().numpy()
    xi = rng.integers(-50, 50, a.cols()).astype(np.float32)
    yi = rng.integers(-50, 50, a.rows()).astype(np.float32)
    axi = (a @ torch.from_numpy(xi).cuda()).cpu().numpy()
    atyi = (torch.from_numpy(yi).cuda() @ a).cpu().numpy()
    for q in range(len(sizes)):
        rs, cs = slice(row0[q], row0[q + 1]), slice(q * C, (q + 1) * C)
        if sizes[q] == 0:
            assert not np.any(aty[cs]) and not np.any(atyi[cs])
            continue
        np.testing.assert_allclose(ax[rs], orc.spmv(idx[q], C, x[cs]), rtol=1e-12, atol=1e-11)
        np.testing.assert_allclose(aty[cs], orc.spmv_t(idx[q], C, y[rs]), rtol=1e-11, atol=1e-10)
        np.testing.assert_array_equal(axi[rs], orc.spmv(idx[q], C, xi[cs].astype(np.float64)).astype(np.float32))
        np.testing.assert_array_equal(atyi[cs], orc.spmv_t(idx[q], C, yi[rs].astype(np.float64)).astype(np.float32))
        with np.errstate(divide="ignore"):
            np.testing.assert_array_equal(jac[cs], orc.jacobi(idx[q], C))


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batched_pcg_reaches_tolerance_per_problem(cuda, orc, precision):
    sizes = [30000, 5000, 12000, 0]
    a, pos, g = _batch(sizes, seed=50, empties=[15, 45, 30, 20])
    C = g.index_space_size
    b = cb.generate_targets(a, 50)
    x, reps, ok = cb.solve_batched(a, b, precision=precision, tol=1e-8, max_iterations=5000)
    assert ok, reps
    row0, idx = _oracle_problems(orc, a, pos)
    bh, xh = b.cpu().numpy(), x.cpu().numpy()
    iters = []
    for q in range(len(sizes)):
        rs = slice(row0[q], row0[q + 1])
        assert reps[q]["converged"] and reps[q]["rel_residual"] <= 1e-8
        if sizes[q] == 0:
            assert reps[q]["iterations"] == 0 and not np.any(xh[q])
            continue
        iters.append(reps[q]["iterations"])
        assert orc.normal_residual(idx[q], C, bh[rs], xh[q]) <= 1.5e-8
        want, _, _ = orc.pcg(idx[q], C, bh[rs], 5000, tol=1e-8, check_every=10)
        pred, pw = orc.spmv(idx[q], C, xh[q]), orc.spmv(idx[q], C, want)
        np.testing.assert_allclose(pred, pw, rtol=0, atol=1e-5 * np.abs(pw).max())
    assert len(set(iters)) > 1  # problems converge (and retire) at different iterations


def test_batched_matches_single_fits(cuda):
    """The batch gives each problem the fit a single solve of it gives."""
    sizes = [20000, 9000]
    a, pos, g = _batch(sizes, seed=60, empties=[22, 38])
    b = cb.generate_targets(a, 60)
    x, reps, ok = cb.solve_batched(a, b, precision="mixed", tol=1e-8)
    assert ok
    row0 = a.problems()
    for q in range(len(sizes)):
        rs = slice(int(row0[q]), int(row0[q + 1]))
        single = cb.MatrixCSR.from_positions(g, pos[rs].contiguous(), "blocked")
        s = cb.PCG(single, b[rs].contiguous(), precision="mixed", tol=1e-8)
        assert s.run()["converged"]
        pb = (single @ x[q].contiguous()).cpu().numpy()
        ps = (single @ s.x()).cpu().numpy()
        np.testing.assert_allclose(pb, ps, rtol=0, atol=1e-5 * np.abs(ps).max())


def test_batched_zero_targets_retire_at_setup(cuda):
    a, pos, g = _batch([3000, 4000], seed=70)
    b = torch.zeros(a.rows(), dtype=torch.float64, device="cuda")
    x, reps, ok = cb.solve_batched(a, b, tol=1e-8)
    assert ok and all(r["iterations"] == 0 for r in reps)
    assert torch.count_nonzero(x) == 0


def test_batched_rejects_bad_sizes(cuda):
    pos = cb.generate_positions(1, 100, 20, 20)
    g = cb.GroupIndexer(SET8, "expanded")
    with pytest.raises(cb.SizeMismatch):
        cb.MatrixCSR.from_positions_batched(g, pos, [50, 49])
    with pytest.raises(cb.CasError):
        cb.MatrixCSR.from_positions_batched(g, pos, [1] * 65 + [35])


def test_fit_weights_batched_host_api(cuda):
    """cas_fit_weights_batched (host buffers) gives the weights of the
    device-resident batched solve."""
    import ctypes as C

    from cassandra_b200 import _lib as L

    sizes = [6000, 2500]
    a, pos, g = _batch(sizes, seed=80, empties=[25, 35])
    b = cb.generate_targets(a, 80)
    x, reps, ok = cb.solve_batched(a, b, precision="mixed", tol=1e-8)
    assert ok
    lib = L.load()
    masks = np.asarray(SET8, np.uint64)
    pos_h = np.ascontiguousarray(pos.cpu().numpy().view(np.uint64))
    sc_h = np.ascontiguousarray(b.cpu().numpy().astype(np.float32))
    rows = np.asarray(sizes, np.int64)
    w = np.empty(a.cols(), np.float32)
    hreps = (L.SolveReport * len(sizes))()
    opts = cb.solve_opts("pcg", "mixed", 1e-8)
    L.check(lib.cas_fit_weights_batched(masks.ctypes.data_as(C.c_void_p), len(masks), L.CAS_INDEX_EXPANDED,
                                        pos_h.ctypes.data_as(C.c_void_p), sc_h.ctypes.data_as(C.c_void_p),
                                        rows.ctypes.data_as(C.c_void_p), len(sizes), C.byref(opts),
                                        w.ctypes.data_as(C.c_void_p), hreps))
    assert all(r.rel_residual <= 1e-8 for r in hreps)
    pw = (a @ torch.from_numpy(w.astype(np.float64)).cuda()).cpu().numpy()
    px = (a @ x.reshape(-1)).cpu().numpy()
    np.testing.assert_allclose(pw, px, rtol=0, atol=1e-4 * np.abs(px).max())


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batched_degenerate_problems(cuda, orc, precision):
    """Rank-deficient problems of the per-stage loop: 60 empties is the start
    position only (all rows equal), 59 and 58 have a handful of distinct rows;
    small problems beside a regular one.  Each reaches the tolerance (or the
    exact solution) and fits like the FP64 oracle."""
    sizes = [20000, 3000, 2500, 1500]
    a, pos, g = _batch(sizes, seed=90, empties=[30, 60, 59, 58])
    C = g.index_space_size
    b = cb.generate_targets(a, 90)
    x, reps, ok = cb.solve_batched(a, b, precision=precision, tol=1e-8, max_iterations=5000)
    assert ok, reps
    row0, idx = _oracle_problems(orc, a, pos)
    bh, xh = b.cpu().numpy(), x.cpu().numpy()
    for q in range(len(sizes)):
        rs = slice(row0[q], row0[q + 1])
        assert orc.normal_residual(idx[q], C, bh[rs], xh[q]) <= 1.5e-8, (q, reps[q])


def test_single_solver_on_identical_rows(cuda, orc):
    """One fit whose rows are all the start position (rank 1)."""
    pos = cb.generate_positions(5, 4000, 60, 60)
    g = cb.GroupIndexer(SET8, "expanded")
    for layout, precision in (("rows", "fp64"), ("blocked", "mixed")):
        a = cb.MatrixCSR.from_positions(g, pos, layout)
        b = cb.generate_targets(a, 5)
        s = cb.PCG(a, b, precision=precision, tol=1e-8, max_iterations=2000)
        rep = s.run()
        assert rep["converged"], (layout, rep)
        idx = orc.group_index(SET8, 1, pos.cpu().numpy().view(np.uint64))
        assert orc.normal_residual(idx, g.index_space_size, b.cpu().numpy(), s.x().cpu().numpy()) <= 1.5e-8


@pytest.mark.parametrize("method,precision,scale", [("lsqr", "mixed", True), ("lsmr", "fp64", True),
                                                    ("lsqr", "fp64", False)])
def test_batched_least_squares_fits(cuda, orc, method, precision, scale):
    """LSQR/LSMR through cas_fit_weights_batched_device: one solver per stage,
    run together on their own streams.  Each stage's weights are bitwise the
    single fit's of that stage with the same options, reach 1e-8 by the
    oracle's FP64 residual, and a stage without rows gets zero weights."""
    sizes = [20000, 0, 9000, 3000]
    empties = [24, 30, 36, 18]
    g = cb.GroupIndexer(SET8, "expanded")
    parts = [cb.generate_positions(90 + q, n, empties[q], empties[q]) for q, n in enumerate(sizes) if n]
    pos = torch.cat(parts)
    a_all = cb.MatrixCSR.from_positions(g, pos, "rows")
    b = cb.generate_targets(a_all, 90)
    kw = dict(method=method, precision=precision, tol=1e-8, max_iterations=40_000, check_every=50,
              scale_columns=scale)
    x, reps, ok = cb.fit_weights_batched(g, pos, b, sizes, **kw)
    assert ok, reps
    assert torch.count_nonzero(x[1]) == 0 and reps[1]["iterations"] == 0
    layout = "blocked" if precision == "mixed" else "rows"
    cls = cb.LSQR if method == "lsqr" else cb.LSMR
    row0 = np.concatenate([[0], np.cumsum(sizes)])
    ph = pos.cpu().numpy().view(np.uint64)
    for q, n in enumerate(sizes):
        if not n:
            continue
        rs = slice(int(row0[q]), int(row0[q + 1]))
        single = cb.MatrixCSR.from_positions(g, pos[rs].contiguous(), layout)
        s = cls(single, b[rs].contiguous(), precision=precision, tol=1e-8, max_iterations=40_000, check_every=50,
                scale_columns=scale)
        rep = s.run()
        assert rep["converged"] and rep["iterations"] == reps[q]["iterations"]
        assert torch.equal(s.x(), x[q])
        idx = orc.group_index(SET8, 1, ph[rs])
        assert orc.normal_residual(idx, g.index_space_size, b[rs].cpu().numpy(), x[q].cpu().numpy()) <= 1.5e-8
