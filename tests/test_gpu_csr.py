"""CSR build and products on the device against the reference's known answers
and the oracle."""
import numpy as np
import pytest
import torch

import cassandra_b200 as cb
from tests.golden.make_golden import SET5, SET8

pytestmark = pytest.mark.gpu


def _csr_from_numpy(idx: np.ndarray, cols: int) -> cb.MatrixCSR:
    return cb.MatrixCSR.from_indices(torch.from_numpy(idx.astype(np.uint32).view(np.int32)).cuda(), cols)


# MathTest/MatrixCSR.cpp:3-55
def test_known_answers(cuda):
    a = _csr_from_numpy(np.array([[0, 1], [1, 2], [3, 3]]), 4)
    assert (a.rows(), a.cols(), a.nnz_per_row) == (3, 4, 2)
    for dt in (torch.float32, torch.float64):
        x = torch.tensor([1, 2, 3, 4], dtype=dt, device="cuda")
        assert (a @ x).tolist() == [3, 5, 8]
        y = torch.tensor([1, 2, 3], dtype=dt, device="cuda")
        assert (y @ a).tolist() == [1, 3, 2, 6]
        assert cb.jacobi_preconditioner_of_ata(a, dt).tolist() == [1, 0.5, 1, 0.25]


def test_size_mismatch(cuda):
    a = _csr_from_numpy(np.array([[0, 1], [1, 2], [3, 3]]), 4)
    with pytest.raises(cb.SizeMismatch):
        a @ torch.zeros(3, dtype=torch.float64, device="cuda")
    with pytest.raises(cb.SizeMismatch):
        torch.zeros(4, dtype=torch.float64, device="cuda") @ a


def test_golden_products(cuda, golden_math):
    g = golden_math
    a = _csr_from_numpy(g["idx"], int(g["cols"]))
    ax = (a @ torch.from_numpy(g["x"]).cuda()).cpu().numpy()
    np.testing.assert_allclose(ax, g["ax"], rtol=2e-6, atol=2e-6)
    aty = (torch.from_numpy(g["y"]).cuda() @ a).cpu().numpy()
    np.testing.assert_allclose(aty, g["aty"], rtol=2e-6, atol=2e-6)
    np.testing.assert_array_equal(cb.jacobi_preconditioner_of_ata(a, torch.float32).cpu().numpy(), g["jacobi"])


def _pattern_system(orc, rows, masks=SET5, mode="reference", seed=3):
    pos = cb.generate_positions(seed, rows, 10, 50)
    g = cb.GroupIndexer(masks, mode)
    a = cb.MatrixCSR.from_positions(g, pos)
    idx = a.indices().cpu().numpy().view(np.uint32)
    return a, idx, g.index_space_size


@pytest.mark.parametrize("mode", ["reference", "expanded"])
def test_csr_from_positions_matches_indexer(cuda, orc, mode):
    pos = cb.generate_positions(8, 20_000, 10, 50)
    g = cb.GroupIndexer(SET8, mode)
    a = cb.MatrixCSR.from_positions(g, pos)
    want = orc.group_index(SET8, 0 if mode == "reference" else 1, pos.cpu().numpy().view(np.uint64))
    np.testing.assert_array_equal(a.indices().cpu().numpy().view(np.uint32), want)


@pytest.mark.parametrize("rows", [1, 777, 50_000])
def test_transposed_is_stable_column_sort(cuda, orc, rows):
    a, idx, cols = _pattern_system(orc, rows, SET8, "expanded")
    col_ptr, row_idx = a.transposed()
    flat = idx.reshape(-1)
    order = np.argsort(flat, kind="stable")
    np.testing.assert_array_equal(row_idx.cpu().numpy().view(np.uint32), (order // idx.shape[1]).astype(np.uint32))
    counts = np.bincount(flat, minlength=cols)
    np.testing.assert_array_equal(col_ptr.cpu().numpy(), np.concatenate([[0], np.cumsum(counts)]))


@pytest.mark.parametrize("mode", ["reference", "expanded"])
def test_products_match_oracle(cuda, orc, mode):
    a, idx, cols = _pattern_system(orc, 30_000, SET8, mode)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(cols)
    y = rng.standard_normal(idx.shape[0])
    got = (a @ torch.from_numpy(x).cuda()).cpu().numpy()
    np.testing.assert_allclose(got, orc.spmv(idx, cols, x), rtol=1e-13, atol=1e-12)
    got = (torch.from_numpy(y).cuda() @ a).cpu().numpy()
    np.testing.assert_allclose(got, orc.spmv_t(idx, cols, y), rtol=1e-12, atol=1e-11)
    with np.errstate(divide="ignore"):
        want = orc.jacobi(idx, cols)
    np.testing.assert_array_equal(cb.jacobi_preconditioner_of_ata(a).cpu().numpy(), want)
    # FP32 products are exact for integer-valued vectors
    xi = rng.integers(-50, 50, cols).astype(np.float32)
    yi = rng.integers(-50, 50, idx.shape[0]).astype(np.float32)
    np.testing.assert_array_equal((a @ torch.from_numpy(xi).cuda()).cpu().numpy(),
                                  orc.spmv(idx, cols, xi.astype(np.float64)).astype(np.float32))
    np.testing.assert_array_equal((torch.from_numpy(yi).cuda() @ a).cpu().numpy(),
                                  orc.spmv_t(idx, cols, yi.astype(np.float64)).astype(np.float32))


def test_products_are_deterministic(cuda, orc):
    a, idx, cols = _pattern_system(orc, 100_000, SET8, "expanded")
    y = torch.randn(idx.shape[0], dtype=torch.float64, device="cuda")
    r1 = (y @ a).cpu().numpy()
    r2 = (y @ a).cpu().numpy()
    assert r1.tobytes() == r2.tobytes()


def test_empty_matrix(cuda):
    g = cb.GroupIndexer(SET5)
    a = cb.MatrixCSR.from_positions(g, torch.empty((0, 2), dtype=torch.int64, device="cuda"))
    assert a.rows() == 0 and a.cols() == g.index_space_size
    x = torch.ones(a.cols(), dtype=torch.float64, device="cuda")
    assert (a @ x).numel() == 0
    assert torch.count_nonzero(torch.empty(0, dtype=torch.float64, device="cuda") @ a) == 0


def test_from_indices_rejects_out_of_range_columns(cuda):
    """Caller-supplied indices are checked (one pass over them) before any
    kernel uses them as addresses: an index >= cols is refused with
    CAS_ERR_INVALID_ARGUMENT, at the first and at the last entry alike."""
    from cassandra_b200 import _lib as L

    for where in (0, -1):
        idx = np.zeros((5000, 7), np.uint32)
        idx.flat[where] = 11
        with pytest.raises(cb.CasError) as e:
            cb.MatrixCSR.from_indices(torch.from_numpy(idx.view(np.int32)).cuda(), 11)
        assert e.value.status == L.CAS_ERR_INVALID_ARGUMENT
    idx[:] = 10
    assert cb.MatrixCSR.from_indices(torch.from_numpy(idx.view(np.int32)).cuda(), 11).cols() == 11
