"""Row-sharded Jacobi-PCG across ranks (one process per GPU).

The fit's rows split naturally: rank k holds a block of rows A_k, b_k, and

    A'A p = sum_k A_k'(A_k p),   A'b = sum_k A_k' b_k,   diag(A'A) = sum_k diag_k,
    p'A'A p = sum_k ||A_k p||^2,

so one PCG iteration needs exactly one collective: a sum all-reduce of the
cols-length partial A_k'A_k p with ||A_k p||^2 appended.  Everything else
(alpha, beta, the x/r/z/p updates, r.z) is computed redundantly and
identically on every rank from the reduced vector, exactly as the
single-GPU PCG does (Math/Solver.h:99-112).  The sparse products of a rank
run on its GPU through the library (``GpuShard``); the collective goes
through torch.distributed (NCCL on GPUs, gloo in the CPU tests, where
``tests/test_parallel.py`` plugs in a host implementation of the same shard
interface to check the communication logic).
"""
from __future__ import annotations

from dataclasses import dataclass

import torch
import torch.distributed as dist


class Shard:
    """What a rank contributes: products with its block of rows."""

    cols: int

    def normal_product(self, p: torch.Tensor) -> tuple[torch.Tensor, float]:
        """(A_k' A_k p, ||A_k p||^2) for this rank's rows."""
        raise NotImplementedError

    def rhs(self) -> torch.Tensor:
        """A_k' b_k."""
        raise NotImplementedError

    def diag(self) -> torch.Tensor:
        """diag(A_k' A_k)."""
        raise NotImplementedError


class GpuShard(Shard):
    """A rank's rows on its GPU (a MatrixCSR and its targets)."""

    def __init__(self, csr, b: torch.Tensor, precision: str = "fp64"):
        from . import jacobi_preconditioner_of_ata

        self.csr = csr
        self.cols = csr.cols()
        self.dtype = torch.float32 if precision == "mixed" else torch.float64
        self.b = b.to(torch.float64)
        d = jacobi_preconditioner_of_ata(csr, torch.float64)
        self._diag = torch.where(torch.isinf(d), torch.zeros_like(d), 1.0 / d)

    def normal_product(self, p):
        q = self.csr.matvec(p.to(self.dtype))
        s = self.csr.rmatvec(q).to(torch.float64)
        return s, float(torch.dot(q.double(), q.double()))

    def rhs(self):
        return self.csr.rmatvec(self.b)

    def diag(self):
        return self._diag


@dataclass
class ShardedResult:
    x: torch.Tensor
    iterations: int
    rel_residual: float
    allreduces: int


def _allreduce(t: torch.Tensor, group) -> torch.Tensor:
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def sharded_pcg(shard: Shard, tol: float = 1e-8, max_iterations: int = 20000, jacobi: bool = True,
                group=None) -> ShardedResult:
    """Jacobi-PCG on sum_k A_k'A_k x = sum_k A_k'b_k from x0 = 0.  Every rank
    calls it with its shard; all ranks return the same x."""
    n_ar = 0
    bn = _allreduce(shard.rhs().to(torch.float64).clone(), group)
    n_ar += 1
    if jacobi:
        diag = _allreduce(shard.diag().to(torch.float64).clone(), group)
        n_ar += 1
        d = 1.0 / diag
        d = torch.where(torch.isfinite(d) & (d != 0), d, torch.ones_like(d))  # DiagonalPreconditioner
    else:
        d = torch.ones_like(bn)
    x = torch.zeros_like(bn)
    r = bn.clone()
    z = d * r
    p = z.clone()
    rz = float(torch.dot(r, z))
    bnorm = float(torch.linalg.vector_norm(bn))
    it = 0
    rel = float(torch.linalg.vector_norm(r)) / bnorm if bnorm > 0 else 0.0
    buf = torch.empty(bn.numel() + 1, dtype=torch.float64, device=bn.device)
    while it < max_iterations and (tol <= 0 or rel > tol):
        s_loc, pap_loc = shard.normal_product(p)
        buf[:-1] = s_loc
        buf[-1] = pap_loc
        _allreduce(buf, group)  # the one collective of the iteration
        n_ar += 1
        s, pap = buf[:-1], float(buf[-1])
        if pap <= 0:
            break
        alpha = rz / pap
        x += alpha * p
        r -= alpha * s
        z = d * r
        rz_new = float(torch.dot(r, z))
        p = z + (rz_new / rz) * p
        rz = rz_new
        it += 1
        rel = float(torch.linalg.vector_norm(r)) / bnorm if bnorm > 0 else 0.0
    return ShardedResult(x=x, iterations=it, rel_residual=rel, allreduces=n_ar)


def split_rows(rows: int, world: int, rank: int, multiple: int = 1) -> tuple[int, int]:
    """Contiguous row range of a rank (boundaries on multiples of `multiple`)."""
    units = (rows + multiple - 1) // multiple
    lo = units * rank // world * multiple
    hi = min(rows, units * (rank + 1) // world * multiple)
    return lo, hi
