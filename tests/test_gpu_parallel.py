"""The row-sharded PCG (cassandra_b200.parallel) on a GPU: GpuShard's products
through the library, the collectives through NCCL, in a process group of
one rank on cuda:0 (every run here has one GPU; the two-rank communication
logic is tested over gloo in tests/test_parallel.py).  Checked against the
single-GPU solver and the FP64 oracle."""
import numpy as np
import pytest
import torch
import torch.distributed as dist

import cassandra_b200 as cb
from cassandra_b200 import parallel as par
from tests.golden.make_golden import SET8

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nccl_group(cuda):
    store = dist.HashStore()
    dist.init_process_group("nccl", store=store, rank=0, world_size=1, device_id=torch.device("cuda", 0))
    yield
    dist.destroy_process_group()


def _system(rows, seed, layout):
    pos = cb.generate_positions(seed, rows, 20, 40)
    g = cb.GroupIndexer(SET8, "expanded")
    a = cb.MatrixCSR.from_positions(g, pos, layout)
    return a, cb.generate_targets(a, seed), pos, g


def test_sharded_fp64_iterates_match_single_gpu_pcg(nccl_group):
    """FP64 products on the rows layout: after 10 iterations x equals the
    single-GPU PCG's (the same recurrences, one collective per iteration)."""
    a, b, _, _ = _system(30_000, 5, "rows")
    res = par.sharded_pcg(par.GpuShard(a, b, "fp64"), tol=0, max_iterations=10)
    s = cb.PCG(a, b, check_every=10)
    s.iterate(10)
    want = s.x()
    assert res.iterations == 10 and res.allreduces == 12
    torch.testing.assert_close(res.x, want, rtol=0, atol=1e-9 * float(want.abs().max()))


def test_sharded_mixed_reaches_tolerance(nccl_group, orc):
    """FP32 products on the blocked layout with FP64 residual replacement at
    chunk boundaries: to 1e-8 by the oracle's FP64 residual, with the
    predictions of the single-GPU mixed solve (a 20,000-row system that FP64
    PCG solves in about 540 iterations; small systems are ill-conditioned:
    at 60,000 rows with this seed FP64 PCG needs 9,650)."""
    a, b, pos, g = _system(20_000, 7, "blocked")
    res = par.sharded_pcg(par.GpuShard(a, b, "mixed"), tol=1e-8, max_iterations=5000)
    assert res.rel_residual <= 1e-8 and res.replacements >= 1
    idx = orc.group_index(SET8, 1, pos.cpu().numpy().view(np.uint64))
    cols = g.index_space_size
    bh = b.cpu().numpy()
    x = res.x.cpu().numpy()
    assert orc.normal_residual(idx, cols, bh, x) <= 1.5e-8
    single = cb.PCG(a, b, precision="mixed", tol=1e-8)
    assert single.run()["converged"]
    pp = orc.spmv(idx, cols, single.x().cpu().numpy())
    assert np.abs(orc.spmv(idx, cols, x) - pp).max() <= 1e-4 * np.abs(pp).max()


def test_rank_blocks_rebuild_the_whole_system(nccl_group):
    """The benchmark's sharded inputs: each rank's block of rows (positions at
    its row numbers, targets drawn for those rows) are the whole system's
    rows, so the ranks' blocks together are the single-GPU system."""
    rows, seed = 3 * 16384 + 777, 11
    a, b, pos, g = _system(rows, seed, "rows")
    for world in (2, 3):
        for rank in range(world):
            lo, hi = par.split_rows(rows, world, rank, int(cb.load().cas_block_rows()))
            p = torch.from_numpy(cb.generate_positions_host(seed, lo, hi - lo, 20, 40).view(np.int64)
                                 .reshape(-1, 2)).cuda()
            assert torch.equal(p, pos[lo:hi])
            ak = cb.MatrixCSR.from_positions(g, p, "rows")
            assert torch.equal(cb.generate_targets(ak, seed, first_row=lo), b[lo:hi])
