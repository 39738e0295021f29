"""PCG / CG / LSQR / LSMR on the device against the FP64 oracle and the reference."""
import numpy as np
import pytest
import torch

import cassandra_b200 as cb
from tests.golden.make_golden import SET5, SET8

pytestmark = pytest.mark.gpu


def _system(rows, masks=SET5, mode="reference", seed=11, lo=20, hi=40):
    pos = cb.generate_positions(seed, rows, lo, hi)
    g = cb.GroupIndexer(masks, mode)
    a = cb.MatrixCSR.from_positions(g, pos)
    b = cb.generate_targets(a, seed)
    idx = a.indices().cpu().numpy().view(np.uint32)
    return a, b, idx, g.index_space_size, pos


def test_pcg_iterates_match_oracle(cuda, orc):
    a, b, idx, cols, _ = _system(4000)
    bh = b.cpu().numpy()
    s = cb.PCG(a, b, check_every=5)
    s.iterate(10)
    want, res, it = orc.pcg(idx, cols, bh, 10)
    got = s.x().cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-10 * np.abs(want).max())
    np.testing.assert_allclose(s.residuum(), res, rtol=1e-8)
    assert s.iterations() == 10


def test_cg_iterates_match_oracle(cuda, orc):
    """Unpreconditioned CG amplifies rounding faster than Jacobi-PCG: iterates
    are pinned after 4 steps and through the predictions after 8."""
    a, b, idx, cols, _ = _system(3000, seed=4)
    bh = b.cpu().numpy()
    s = cb.CG(a, b, check_every=2)
    s.iterate(4)
    want, res, _ = orc.pcg(idx, cols, bh, 4, jacobi=False)
    np.testing.assert_allclose(s.x().cpu().numpy(), want, rtol=0, atol=1e-10 * np.abs(want).max())
    s.iterate(4)
    want, res, _ = orc.pcg(idx, cols, bh, 8, jacobi=False)
    pw = orc.spmv(idx, cols, want)
    np.testing.assert_allclose(orc.spmv(idx, cols, s.x().cpu().numpy()), pw, rtol=0, atol=1e-6 * np.abs(pw).max())


def test_lsqr_iterates_match_oracle(cuda, orc):
    a, b, idx, cols, _ = _system(3000, seed=5)
    bh = b.cpu().numpy()
    s = cb.LSQR(a, b, check_every=5)
    s.iterate(5)
    want, res, _ = orc.lsqr(idx, cols, bh, 5)
    np.testing.assert_allclose(s.x().cpu().numpy(), want, rtol=0, atol=1e-9 * np.abs(want).max())
    np.testing.assert_allclose(s.residuum(), res, rtol=1e-9)


def test_lsmr_iterates_match_oracle(cuda, orc):
    """LSMR (Math/Solver.h:222-287) against the oracle's FP64 restatement.
    Like LSQR, unpreconditioned LSMR amplifies the rounding differences of
    differently ordered sums about 15-fold per step on this system (device
    vs oracle, measured: 1e-11 of the largest weight after 5 steps, 2e-8
    after 8, 5e-6 after 10, for LSQR and LSMR alike), so the iterates are
    pinned after 5 steps and the predictions A x after 8; Residuum() is 0 as
    in the reference."""
    a, b, idx, cols, _ = _system(3000, seed=5)
    bh = b.cpu().numpy()
    s = cb.LSMR(a, b, check_every=5)
    s.iterate(5)
    want, _, _ = orc.lsmr(idx, cols, bh, 5)
    np.testing.assert_allclose(s.x().cpu().numpy(), want, rtol=0, atol=1e-9 * np.abs(want).max())
    assert s.residuum() == 0.0
    s.iterate(3)
    want, _, _ = orc.lsmr(idx, cols, bh, 8)
    pw = orc.spmv(idx, cols, want)
    np.testing.assert_allclose(orc.spmv(idx, cols, s.x().cpu().numpy()), pw, rtol=0, atol=1e-6 * np.abs(pw).max())
    assert s.iterations() == 8


@pytest.mark.parametrize("layout,precision", [("rows", "fp64"), ("blocked", "fp64"), ("blocked", "mixed")])
def test_lsmr_reaches_tolerance(cuda, orc, layout, precision):
    """LSMR to 1e-8 in both precisions; the mixed solve restarts from the
    FP64 residual (an outer refinement step) when its recursive estimate has
    dropped 1e4-fold, like mixed LSQR."""
    pos = cb.generate_positions(8, 3000, 20, 40)
    g = cb.GroupIndexer(SET5, "reference")
    a = cb.MatrixCSR.from_positions(g, pos, layout)
    b = cb.generate_targets(a, 8)
    idx = orc.group_index(SET5, 0, pos.cpu().numpy().view(np.uint64))
    tol = 1e-8
    s = cb.LSMR(a, b, precision=precision, tol=tol, max_iterations=60_000, check_every=50)
    rep = s.run()
    assert rep["converged"], rep
    assert rep["residuum"] == 0.0
    assert orc.normal_residual(idx, g.index_space_size, b.cpu().numpy(), s.x().cpu().numpy()) <= 1.5 * tol


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("mode", ["reference", "expanded"])
def test_pcg_reaches_tolerance(cuda, orc, precision, mode):
    a, b, idx, cols, _ = _system(20_000, SET8, mode, seed=21)
    s = cb.PCG(a, b, precision=precision, tol=1e-8, max_iterations=5000)
    rep = s.run()
    assert rep["converged"], rep
    assert rep["rel_residual"] <= 1e-8
    x = s.x().cpu().numpy()
    bh = b.cpu().numpy()
    # independent FP64 check on the host
    assert orc.normal_residual(idx, cols, bh, x) <= 1.5e-8
    # same least-squares fit as the oracle's FP64 PCG run to the same tolerance
    want, _, _ = orc.pcg(idx, cols, bh, 5000, tol=1e-8, check_every=10)
    pred, pw = orc.spmv(idx, cols, x), orc.spmv(idx, cols, want)
    np.testing.assert_allclose(pred, pw, rtol=0, atol=1e-5 * np.abs(pw).max())


def test_cpu_runnable_workload_200_steps(cuda, orc):
    """The CPU-runnable workload: 100,000 positions of random play to exactly
    30 empties, the 5 masks in expanded mode (C = 150,903 > rows, K = 40),
    Jacobi-PCG from x = 0 in plain FP64.  This system is underdetermined and
    the iteration chaotic: a 1e-15 relative change of b moves the predictions
    by 2e-4 after 30 steps and 1e-3 after 200, and the 200-step normal
    residual anywhere between 1.7e-5 and 2e-4 (six oracle runs).  So the
    predictions are pinned after 10 steps and the 200-step iterate through
    the order of its normal-equation residual."""
    a, b, idx, cols, _ = _system(100_000, SET5, "expanded", seed=3, lo=30, hi=30)
    assert (cols, idx.shape[1]) == (150_903, 40)
    bh = b.cpu().numpy()
    s = cb.PCG(a, b, check_every=10)
    s.iterate(10)
    want, _, _ = orc.pcg(idx, cols, bh, 10)
    pw = orc.spmv(idx, cols, want)
    np.testing.assert_allclose(orc.spmv(idx, cols, s.x().cpu().numpy()), pw, rtol=0, atol=1e-8 * np.abs(pw).max())
    s.iterate(190)
    want, _, _ = orc.pcg(idx, cols, bh, 200)
    res_got = orc.normal_residual(idx, cols, bh, s.x().cpu().numpy())
    res_want = orc.normal_residual(idx, cols, bh, want)
    assert 1e-6 < res_got < 1e-3 and res_got <= 20 * res_want, (res_got, res_want)


def test_lsqr_reaches_tolerance(cuda, orc):
    a, b, idx, cols, _ = _system(3000, SET5, seed=8)
    s = cb.LSQR(a, b, tol=1e-8, max_iterations=50_000, check_every=100)
    rep = s.run()
    assert rep["converged"], rep
    assert orc.normal_residual(idx, cols, b.cpu().numpy(), s.x().cpu().numpy()) <= 1.5e-8


def test_fit_weights_host_api_matches_reference_fitweights(cuda, ref):
    """cas_fit_weights with the reference's FitWeights(pattern, pos, 10): same
    10 Jacobi-PCG steps; the reference runs them in FP32."""
    import ctypes as C

    pos = cb.generate_positions_host(17, 0, 5000, 20, 40)
    rng = np.random.default_rng(17)
    scores = (2 * rng.integers(-16, 17, len(pos))).astype(np.float32)
    w, rep = cb.fit_weights(SET5, pos, scores, mode="reference", tol=0, max_iterations=10, check_every=10)
    assert rep["iterations"] == 10
    m = np.asarray(SET5, np.uint64)
    cols = np.zeros(1, np.int64)
    lib = ref.ref_lib()
    k = lib.ref_group_info(m.ctypes.data_as(C.c_void_p), len(m), cols.ctypes.data_as(C.c_void_p), None)
    idx = np.empty((len(pos), k), np.uint32)
    lib.ref_group_index(m.ctypes.data_as(C.c_void_p), len(m), pos.ctypes.data_as(C.c_void_p), len(pos),
                        idx.ctypes.data_as(C.c_void_p))
    want = np.empty(int(cols[0]), np.float32)
    res = C.c_float()
    lib.ref_pcg(k, len(pos), int(cols[0]), idx.ctypes.data_as(C.c_void_p), scores.ctypes.data_as(C.c_void_p), 10,
                want.ctypes.data_as(C.c_void_p), C.byref(res))
    np.testing.assert_allclose(w, want, rtol=0, atol=2e-4 * np.abs(want).max())


def test_solver_size_mismatch(cuda):
    a, b, idx, cols, _ = _system(100)
    with pytest.raises(cb.SizeMismatch):
        cb.PCG(a, b[:-1])
    with pytest.raises(cb.SizeMismatch):
        cb.PCG(a, b, x0=torch.zeros(cols + 1, dtype=torch.float64, device="cuda"))


def test_zero_rhs_converges_immediately(cuda):
    a, b, idx, cols, _ = _system(500)
    s = cb.PCG(a, torch.zeros_like(b), tol=1e-8)
    rep = s.run()
    assert rep["converged"] and rep["iterations"] == 0
    assert torch.count_nonzero(s.x()) == 0


@pytest.mark.parametrize("method", ["lsqr", "lsmr"])
def test_scaled_least_squares_iterates_match_oracle(cuda, orc, method):
    """LSQR/LSMR with column scaling (scale_columns: iterating on A S, S =
    diag(A'A)^-1/2) against the oracle's scaled restatement, plain FP64 on the
    rows layout: iterates after 5 steps, predictions after 8."""
    a, b, idx, cols, _ = _system(3000, seed=5)
    bh = b.cpu().numpy()
    cls = cb.LSQR if method == "lsqr" else cb.LSMR
    fn = orc.lsqr if method == "lsqr" else orc.lsmr
    s = cls(a, b, check_every=5, scale_columns=True)
    s.iterate(5)
    want, _, _ = fn(idx, cols, bh, 5, scale=True)
    np.testing.assert_allclose(s.x().cpu().numpy(), want, rtol=0, atol=1e-9 * np.abs(want).max())
    s.iterate(3)
    want, _, _ = fn(idx, cols, bh, 8, scale=True)
    pw = orc.spmv(idx, cols, want)
    np.testing.assert_allclose(orc.spmv(idx, cols, s.x().cpu().numpy()), pw, rtol=0, atol=1e-6 * np.abs(pw).max())


@pytest.mark.parametrize("scale", [False, True])
@pytest.mark.parametrize("method", ["lsqr", "lsmr"])
@pytest.mark.parametrize("layout,precision", [("rows", "fp64"), ("blocked", "mixed")])
def test_least_squares_reach_1e8_on_fit_system(cuda, orc, method, scale, layout, precision):
    """LSQR and LSMR, unscaled (the reference's methods) and column-scaled, to
    1e-8 on a 20,000-row 8-pattern expanded system: the FP64 oracle's
    residual of the returned x meets the tolerance and its predictions are
    the PCG least-squares fit's."""
    pos = cb.generate_positions(31, 20_000, 20, 40)
    g = cb.GroupIndexer(SET8, "expanded")
    a = cb.MatrixCSR.from_positions(g, pos, layout)
    b = cb.generate_targets(a, 31)
    idx = orc.group_index(SET8, 1, pos.cpu().numpy().view(np.uint64))
    cols = g.index_space_size
    cls = cb.LSQR if method == "lsqr" else cb.LSMR
    s = cls(a, b, precision=precision, tol=1e-8, max_iterations=40_000, check_every=100, scale_columns=scale)
    rep = s.run()
    assert rep["converged"], rep
    if precision == "mixed":
        assert rep["refinements"] >= 1
    bh = b.cpu().numpy()
    x = s.x().cpu().numpy()
    assert orc.normal_residual(idx, cols, bh, x) <= 1.5e-8
    xp, _, _ = orc.pcg(idx, cols, bh, 5000, tol=1e-10, check_every=10)
    pp = orc.spmv(idx, cols, xp)
    assert np.abs(orc.spmv(idx, cols, x) - pp).max() <= 1e-4 * np.abs(pp).max()


@pytest.mark.parametrize("method,layout,precision", [("pcg", "rows", "fp64"), ("pcg", "blocked", "mixed"),
                                                     ("lsqr", "blocked", "mixed"), ("lsmr", "rows", "fp64")])
def test_checkpoint_resumes_bitwise(cuda, method, layout, precision):
    """cas_solver_save_state / cas_solver_load_state: a solver created on the
    same system that loads a checkpoint taken after 30 iterations produces,
    over 40 more (FP64 residual replacements or restarts of the mixed solvers
    included), bitwise the iterate of the solver that was never stopped; the
    checkpoint does not load into a solver of another method or precision."""
    pos = cb.generate_positions(23, 20_000, 20, 40)
    g = cb.GroupIndexer(SET8, "expanded")
    a = cb.MatrixCSR.from_positions(g, pos, layout)
    b = cb.generate_targets(a, 23)
    cls = {"pcg": cb.PCG, "lsqr": cb.LSQR, "lsmr": cb.LSMR}[method]
    kw = dict(precision=precision, tol=1e-12, check_every=10)
    s1 = cls(a, b, **kw)
    s1.iterate(30)
    state = s1.save_state()
    s1.iterate(40)
    want = s1.x()
    s2 = cls(a, b, **kw)
    s2.iterate(3)  # a different state, overwritten by the load
    s2.load_state(bytes(state))
    assert s2.iterations() == 30
    s2.iterate(40)
    assert s2.iterations() == s1.iterations() == 70
    assert torch.equal(s2.x(), want)
    other = cb.CG(a, b, precision=precision) if method != "pcg" else cb.PCG(a, b, precision="fp64" if precision == "mixed" else "mixed")
    with pytest.raises(cb.CasError):
        other.load_state(state)
    with pytest.raises(cb.CasError):
        s2.load_state(state[:100])


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_host_fit_equals_device_fit(cuda, precision):
    """cas_fit_weights (host buffers: positions uploaded in row chunks, each
    indexed as soon as it lands; scores uploaded while the layout builds)
    returns bitwise the weights of cas_fit_weights_device on the same inputs,
    on a row count that splits into neither whole chunks nor whole blocks."""
    import ctypes as C

    from cassandra_b200 import _lib as L

    rows = 3 * 16384 + 4099
    pos = cb.generate_positions_host(29, 0, rows, 20, 40)
    g = cb.GroupIndexer(SET8, "expanded")
    d_pos = torch.from_numpy(pos.view(np.int64).reshape(-1, 2)).cuda()
    scores = cb.generate_targets(cb.MatrixCSR.from_positions(g, d_pos, "rows"), 29).cpu().numpy().astype(np.float32)
    w_host, rep = cb.fit_weights(SET8, pos, scores, mode="expanded", precision=precision, tol=1e-8)
    lib = L.load()
    d_sc = torch.from_numpy(scores.astype(np.float64)).cuda()
    w = torch.empty(g.index_space_size, dtype=torch.float64, device="cuda")
    drep = L.SolveReport()
    opts = cb.solve_opts("pcg", precision, 1e-8)
    L.check(lib.cas_fit_weights_device(g.handle, C.c_void_p(d_pos.data_ptr()), C.c_void_p(d_sc.data_ptr()), rows,
                                       C.byref(opts), C.c_void_p(w.data_ptr()), C.byref(drep),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    assert drep.iterations == rep["iterations"]
    np.testing.assert_array_equal(w_host, w.cpu().numpy().astype(np.float32))
    assert rep["converged"], rep
