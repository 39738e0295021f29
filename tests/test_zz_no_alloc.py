"""The allocation-free product cas_spmv_norm_noalloc, called through the C ABI
the way a caller that cannot allocate device memory would: with its own
buffers, twice in a row, checked against the regular entry point cas_spmv
and the FP64 oracle (y) and against y.y of that result (||y||^2); at the
exact row capacity of its fixed scratch; and with an index out of range.

Such callers own all device memory themselves (another allocator, a fixed
budget) or run where cudaMalloc may not be called, so the entry point keeps
its partial sums in a fixed array inside the library instead of allocating.
This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest
import torch

import cassandra_b200 as cb
from cassandra_b200 import _lib as L
from tests.golden.make_golden import SET8

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_matches_regular_entry_point_twice(cuda, orc):
    lib = L.load()
    rows = 70_001  # 35 CTAs, the last one partial
    pos = cb.generate_positions(3, rows, 10, 50)
    g = cb.GroupIndexer(SET8, "expanded")
    a = cb.MatrixCSR.from_positions(g, pos, "rows")
    idx = lib.cas_csr_indices(a.handle)
    cols, k = a.cols(), a.nnz_per_row
    idx_host = a.indices().cpu().numpy().view(np.uint32).reshape(rows, k)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # caller-owned buffers, allocated before the calls
    y = torch.empty(rows, dtype=torch.float64, device="cuda")
    y_ref = torch.empty(rows, dtype=torch.float64, device="cuda")
    n2 = torch.empty(1, dtype=torch.float64, device="cuda")
    for trial in range(2):
        x = torch.randn(cols, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(trial))
        L.check(lib.cas_spmv_norm_noalloc(C.c_void_p(idx), k, rows, cols, _p(x), _p(y), _p(n2), stream))
        L.check(lib.cas_spmv(a.handle, L.CAS_F64, _p(x), _p(y_ref), stream))
        torch.cuda.synchronize()
        yh, yr = y.cpu().numpy(), y_ref.cpu().numpy()
        np.testing.assert_allclose(yh, yr, rtol=1e-13, atol=1e-12)
        np.testing.assert_allclose(yh, orc.spmv(idx_host, cols, x.cpu().numpy()), rtol=1e-13, atol=1e-12)
        want = float(np.dot(yr, yr))
        assert abs(float(n2.item()) - want) <= 1e-12 * want


def test_noalloc_at_its_row_capacity(cuda):
    """Exactly cas_spmv_norm_noalloc_max_rows() rows (every one of the
    8192 partials of the fixed scratch in use, the finishing sum over all of
    them), one index per row: y is x gathered, ||y||^2 is y.y."""
    lib = L.load()
    rows = lib.cas_spmv_norm_noalloc_max_rows()
    cols = 1000
    gen = torch.Generator("cuda").manual_seed(7)
    idx = torch.randint(0, cols, (rows,), dtype=torch.int32, device="cuda", generator=gen)
    x = torch.randn(cols, dtype=torch.float64, device="cuda", generator=gen)
    y = torch.empty(rows, dtype=torch.float64, device="cuda")
    n2 = torch.empty(1, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    L.check(lib.cas_spmv_norm_noalloc(_p(idx), 1, rows, cols, _p(x), _p(y), _p(n2), stream))
    torch.cuda.synchronize()
    want_y = x[idx.long()]
    assert torch.equal(y, want_y)
    want = float(torch.dot(want_y, want_y))
    assert abs(float(n2.item()) - want) <= 1e-12 * want
    del idx, x, y, want_y


def test_noalloc_never_reads_through_an_out_of_range_index(cuda):
    """The call is asynchronous, so a column index >= cols cannot come back
    as a status: it is not read through, its row's y and the norm are NaN,
    and the other rows are unaffected."""
    lib = L.load()
    rows, k, cols = 5000, 4, 50
    idx_h = np.random.default_rng(1).integers(0, cols, (rows, k)).astype(np.uint32)
    idx_h[1234, 2] = 1 << 30  # far outside x
    idx = torch.from_numpy(idx_h.view(np.int32)).cuda()
    x = torch.arange(cols, dtype=torch.float64, device="cuda")
    y = torch.empty(rows, dtype=torch.float64, device="cuda")
    n2 = torch.empty(1, dtype=torch.float64, device="cuda")
    L.check(lib.cas_spmv_norm_noalloc(_p(idx), k, rows, cols, _p(x), _p(y), _p(n2), None))
    torch.cuda.synchronize()
    yh = y.cpu().numpy()
    assert np.isnan(yh[1234]) and np.isnan(float(n2.item()))
    good = np.ones(rows, bool)
    good[1234] = False
    np.testing.assert_array_equal(yh[good], idx_h[good].astype(np.float64).sum(axis=1))


def test_noalloc_rejects_rows_beyond_its_scratch(cuda):
    lib = L.load()
    limit = lib.cas_spmv_norm_noalloc_max_rows()
    assert limit == 16_777_216
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    st = lib.cas_spmv_norm_noalloc(_p(buf), 1, limit + 1, 1, _p(buf), _p(buf), _p(buf), None)
    assert st == L.CAS_ERR_INVALID_ARGUMENT
    assert "16,777,216" in L.last_error()


def test_noalloc_empty_matrix(cuda):
    lib = L.load()
    n2 = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
    L.check(lib.cas_spmv_norm_noalloc(None, 8, 0, 10, None, None, _p(n2), None))
    torch.cuda.synchronize()
    assert float(n2.item()) == 0.0
