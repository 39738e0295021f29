"""The allocation-free product cas_spmv_norm_noalloc, called through the C ABI
the way a caller that cannot allocate device memory would: with its own
buffers, twice in a row, checked against the regular entry point cas_spmv
(y) and against y.y of that result (||y||^2).

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


def test_noalloc_matches_regular_entry_point_twice(cuda):
    lib = L.load()
    rows = 70_001  # 35 CTAs, the last one partial
    pos = cb.generate_positions(3, rows, 10, 50)
    g = cb.GroupIndexer(SET8, "expanded")
    a = cb.MatrixCSR.from_positions(g, pos, "rows")
    idx = lib.cas_csr_indices(a.handle)
    cols, k = a.cols(), a.nnz_per_row
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
        want = float(np.dot(yr, yr))
        assert abs(float(n2.item()) - want) <= 1e-12 * want


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
