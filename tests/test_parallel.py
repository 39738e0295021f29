"""Row-sharded PCG with world_size 2 over gloo on CPU: the communication
logic of cassandra_b200.parallel with a host implementation of the shard
interface (the oracle's products), checked against the single-process
oracle PCG.  GPU shards use the same driver with NCCL."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cassandra_b200 import parallel as par


class HostShard(par.Shard):
    """Test double of a rank's rows: products by the C oracle on the host."""

    def __init__(self, idx, cols, b):
        import oracle

        self.o, self.idx, self.cols, self.b = oracle, idx, cols, b

    def normal_product(self, p):
        q = self.o.spmv(self.idx, self.cols, p.numpy())
        return torch.from_numpy(self.o.spmv_t(self.idx, self.cols, q)), float(q @ q)

    def rhs(self):
        return torch.from_numpy(self.o.spmv_t(self.idx, self.cols, self.b))

    def diag(self):
        with np.errstate(divide="ignore"):
            d = self.o.jacobi(self.idx, self.cols)
        return torch.from_numpy(np.where(np.isinf(d), 0.0, 1.0 / d))


def _system():
    import oracle
    import cassandra_b200 as cb

    pos = cb.generate_positions_host(21, 0, 4000, 20, 40)
    masks = cb.PATTERNS_5
    idx = oracle.group_index(masks, 0, pos)
    cols, _ = oracle.group_info(masks, 0)
    rng = np.random.default_rng(21)
    w = rng.normal(0, 0.5, cols)
    b = np.clip(2 * np.rint((oracle.spmv(idx, cols, w) + rng.normal(0, 4, len(pos))) / 2), -64, 64)
    return idx, cols, b


def _worker(rank, world, port, iters, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        idx, cols, b = _system()
        lo, hi = par.split_rows(len(b), world, rank)
        res = par.sharded_pcg(HostShard(idx[lo:hi], cols, b[lo:hi]), tol=0, max_iterations=iters)
        q.put((rank, res.x.numpy(), res.iterations, res.allreduces))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [1, 2])
def test_sharded_pcg_matches_single_process(world):
    import oracle

    iters = 8
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, iters, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    idx, cols, b = _system()
    want, _, _ = oracle.pcg(idx, cols, b, iters)
    xs = {r: x for r, x, _, _ in out}
    for r, x, it, n_ar in out:
        assert it == iters
        assert n_ar == iters + 2  # one per iteration + A'b + diag
        np.testing.assert_allclose(x, want, rtol=0, atol=1e-9 * np.abs(want).max())
    if world == 2:
        np.testing.assert_array_equal(xs[0], xs[1])  # replicated state is identical on every rank


def test_split_rows_covers_everything():
    for rows in (1, 7, 16384, 100_003):
        for world in (1, 2, 3, 8):
            ranges = [par.split_rows(rows, world, r, 16384) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == rows
            for (a, b), (c, d) in zip(ranges, ranges[1:]):
                assert b == c and a <= b
