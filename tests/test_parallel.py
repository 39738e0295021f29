"""Row-sharded PCG with world_size 2 over gloo on CPU: the communication
logic of cassandra_b200.parallel with a host implementation of the shard
interface (the oracle's products), checked against the single-process
oracle PCG.  GPU shards use the same driver with NCCL."""
import os
import queue
import socket
import time

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cassandra_b200 import parallel as par


class HostShard(par.Shard):
    """Test double of a rank's rows: products by the C oracle on the host.
    mixed=True rounds the products' inputs and outputs to FP32, as the GPU
    shard's FP32 products do."""

    def __init__(self, idx, cols, b, mixed=False):
        import oracle

        self.o, self.idx, self.cols, self.b, self.mixed = oracle, idx, cols, b, mixed

    def _r(self, v):
        return v.astype(np.float32).astype(np.float64) if self.mixed else v

    def normal_product(self, p):
        q = self._r(self.o.spmv(self.idx, self.cols, self._r(p.numpy())))
        s = self._r(self.o.spmv_t(self.idx, self.cols, q))
        return torch.from_numpy(s), torch.tensor(float(q @ q), dtype=torch.float64)

    def residual_product(self, x):
        r = self.b - self.o.spmv(self.idx, self.cols, x.numpy())
        return torch.from_numpy(self.o.spmv_t(self.idx, self.cols, r))

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


def _worker(rank, world, port, iters, q, tol=0.0, mixed=False):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        idx, cols, b = _system()
        lo, hi = par.split_rows(len(b), world, rank)
        res = par.sharded_pcg(HostShard(idx[lo:hi], cols, b[lo:hi], mixed), tol=tol, max_iterations=iters,
                              check_every=25)
        q.put((rank, res.x.numpy(), res.iterations, res.allreduces, res.rel_residual, res.replacements))
    finally:
        dist.destroy_process_group()


def _run(world, iters, tol=0.0, mixed=False):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, iters, q, tol, mixed)) for r in range(world)]
    for p in procs:
        p.start()
    out, deadline = [], time.time() + 300
    while len(out) < world:
        try:
            out.append(q.get(timeout=2))
        except queue.Empty:
            failed = [p.exitcode for p in procs if p.exitcode not in (None, 0)]
            assert not failed, f"a rank exited with {failed}"
            assert time.time() < deadline, "ranks did not finish"
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [1, 2])
def test_sharded_pcg_matches_single_process(world):
    import oracle

    iters = 8
    out = _run(world, iters)
    idx, cols, b = _system()
    want, _, _ = oracle.pcg(idx, cols, b, iters)
    xs = {r: x for r, x, *_ in out}
    for r, x, it, n_ar, _, _ in out:
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


@pytest.mark.parametrize("mixed", [False, True])
def test_sharded_pcg_reaches_tolerance(mixed):
    """To 1e-8 over two ranks, with FP64 products and with FP32-rounded ones
    (which need the chunk-boundary replacements by the FP64 true residual):
    the oracle's residual of the returned x meets the tolerance and both
    ranks return the same x."""
    import oracle

    out = _run(2, 5000, tol=1e-8, mixed=mixed)
    idx, cols, b = _system()
    xs = [x for _, x, *_ in out]
    np.testing.assert_array_equal(xs[0], xs[1])
    for _, x, it, n_ar, rel, repl in out:
        assert rel <= 1e-8 and it < 5000
        assert oracle.normal_residual(idx, cols, b, x) <= 1.5e-8
        if mixed:
            assert repl >= 1
