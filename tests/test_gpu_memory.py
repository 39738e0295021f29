"""The library's memory cache: freed layouts and solvers leave their blocks
in the cache, the next objects reuse them (with results unchanged), and
cas_release_cached_memory returns everything."""
import numpy as np
import pytest
import torch

import cassandra_b200 as cb
from cassandra_b200 import _lib as L
from tests.golden.make_golden import SET8

pytestmark = pytest.mark.gpu


def _fit(pos, g, b):
    a = cb.MatrixCSR.from_positions(g, pos, "blocked")
    s = cb.PCG(a, b, precision="mixed", tol=1e-8)
    rep = s.run()
    x = s.x()
    del s, a
    return x, rep


def test_freed_objects_are_cached_and_reused(cuda):
    lib = L.load()
    lib.cas_release_cached_memory()
    assert lib.cas_cached_memory() == 0
    pos = cb.generate_positions(11, 50_000, 20, 40)
    g = cb.GroupIndexer(SET8, "expanded")
    b = cb.generate_targets(cb.MatrixCSR.from_positions(g, pos, "rows"), 11)
    torch.cuda.synchronize()
    x1, r1 = _fit(pos, g, b)
    torch.cuda.synchronize()
    held = lib.cas_cached_memory()
    assert held > 50_000 * 64 * 6  # the layout (A16 + G32) went back to the cache
    x2, r2 = _fit(pos, g, b)  # the same shapes: served from the cache
    torch.cuda.synchronize()
    assert r1["converged"] and r2["converged"] and r1["iterations"] == r2["iterations"]
    assert x1.cpu().numpy().tobytes() == x2.cpu().numpy().tobytes()
    assert lib.cas_cached_memory() <= held * 1.05
    lib.cas_release_cached_memory()
    assert lib.cas_cached_memory() == 0


def test_reused_blocks_do_not_leak_old_contents(cuda, orc):
    """A layout built into blocks another layout freed gives the products of
    its own data."""
    lib = L.load()
    g = cb.GroupIndexer(SET8, "expanded")
    pa = cb.generate_positions(21, 30_000, 15, 25)
    a = cb.MatrixCSR.from_positions(g, pa, "blocked")
    del a
    torch.cuda.synchronize()
    assert lib.cas_cached_memory() > 0
    pb = cb.generate_positions(22, 30_000, 35, 45)
    bm = cb.MatrixCSR.from_positions(g, pb, "blocked")
    idx = orc.group_index(SET8, 1, pb.cpu().numpy().view(np.uint64))
    y = np.random.default_rng(1).integers(-50, 50, 30_000).astype(np.float32)
    got = (torch.from_numpy(y).cuda() @ bm).cpu().numpy()
    np.testing.assert_array_equal(got, orc.spmv_t(idx, g.index_space_size, y.astype(np.float64)).astype(np.float32))
