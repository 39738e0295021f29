"""Row-sharded Jacobi-PCG across ranks (one process per GPU).

The fit's rows split naturally: rank k holds a block of rows A_k, b_k, and

    A'A p = sum_k A_k'(A_k p),   A'b = sum_k A_k' b_k,   diag(A'A) = sum_k diag_k,
    p'A'A p = sum_k ||A_k p||^2,

so one PCG iteration needs exactly one collective: a sum all-reduce of the
cols-length partial A_k'A_k p with ||A_k p||^2 appended.  Everything else
(alpha, beta, the x/r/z/p updates, r.z) is computed redundantly and
identically on every rank from the reduced vector, as the single-GPU PCG
does (Math/Solver.h:99-112).  The replicated state and every scalar stay on
the device: an iteration reads nothing back to the host, and the residual is
read once per chunk of `check_every` iterations.

With FP32 products (a GpuShard of precision "mixed") the recursive residual
drifts from the true one, so it is replaced by the true residual
A'(b - A x), computed in FP64 (one more all-reduce of a cols-length
vector), once it has dropped by REPLACE_DROP since the last replacement,
after refine_every iterations, or when it meets the tolerance (checked at
chunk boundaries, every check_every iterations); a replacement that finds
the recursive residual more than 10 % off restarts the direction, and
convergence is declared on the true residual only -- the single-GPU mixed
solver's reliable updating, at chunk granularity.

Every decision (stop, replace, restart) is taken from all-reduced values, so
every rank takes the same collective steps in the same order.  The sparse
products of a rank run on its GPU through the library (``GpuShard``); the
collectives go through torch.distributed (NCCL on GPUs, gloo in the CPU
tests, where ``tests/test_parallel.py`` plugs in a host implementation of
the same shard interface to check the communication logic).
"""
from __future__ import annotations

from dataclasses import dataclass

import torch
import torch.distributed as dist


class Shard:
    """What a rank contributes: products with its block of rows."""

    cols: int
    mixed: bool = False  # FP32 products (the recursive residual needs replacing)

    def normal_product(self, p: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """(A_k' A_k p, ||A_k p||^2) for this rank's rows, FP64, the norm as a
        0-d tensor on the shard's device."""
        raise NotImplementedError

    def residual_product(self, x: torch.Tensor) -> torch.Tensor:
        """A_k'(b_k - A_k x) in FP64."""
        raise NotImplementedError

    def rhs(self) -> torch.Tensor:
        """A_k' b_k."""
        raise NotImplementedError

    def diag(self) -> torch.Tensor:
        """diag(A_k' A_k)."""
        raise NotImplementedError


class GpuShard(Shard):
    """A rank's rows on its GPU (a MatrixCSR and its targets).  precision
    "mixed" runs the iteration's products in FP32 (on the blocked layout when
    the CSR has it), "fp64" in FP64."""

    def __init__(self, csr, b: torch.Tensor, precision: str = "fp64"):
        from . import jacobi_preconditioner_of_ata

        self.csr = csr
        self.cols = csr.cols()
        self.mixed = precision == "mixed"
        self.dtype = torch.float32 if self.mixed else torch.float64
        self.b = b.to(torch.float64)
        d = jacobi_preconditioner_of_ata(csr, torch.float64)
        self._diag = torch.where(torch.isinf(d), torch.zeros_like(d), 1.0 / d)

    def normal_product(self, p):
        q = self.csr.matvec(p.to(self.dtype))
        s = self.csr.rmatvec(q).to(torch.float64)
        qd = q.to(torch.float64)
        return s, torch.dot(qd, qd)

    def residual_product(self, x):
        return self.csr.rmatvec(self.b - self.csr.matvec(x.to(torch.float64)))

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
    replacements: int = 0


# a replacement that finds the recursive residual this far off restarts the direction
RESTART_DEVIATION = 0.1
# FP32 products: the recursive residual is replaced once it has dropped this
# much since the last replacement (before FP32 drift relative to it grows)
REPLACE_DROP = 1e-3


def _allreduce(t: torch.Tensor, group) -> torch.Tensor:
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def sharded_pcg(shard: Shard, tol: float = 1e-8, max_iterations: int = 20000, jacobi: bool = True,
                group=None, check_every: int = 10, refine_every: int = 50) -> ShardedResult:
    """Jacobi-PCG on sum_k A_k'A_k x = sum_k A_k'b_k from x0 = 0.  Every rank
    calls it with its shard; all ranks return the same x.  tol <= 0 runs
    exactly max_iterations iterations with no checks (one all-reduce per
    iteration after the two of the set-up)."""
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
    rz = torch.dot(r, z)
    bn2 = torch.dot(bn, bn)
    zero = torch.zeros((), dtype=torch.float64, device=bn.device)
    buf = torch.empty(bn.numel() + 1, dtype=torch.float64, device=bn.device)
    it, replacements = 0, 0
    chunk = check_every if tol > 0 and check_every > 0 else max_iterations

    def rel_of(v: torch.Tensor) -> float:
        b2 = float(bn2)
        vv = float(torch.dot(v, v))
        return (vv / b2) ** 0.5 if b2 > 0 else vv ** 0.5

    rel = rel_of(r)
    if tol > 0 and rel <= tol:
        return ShardedResult(x=x, iterations=0, rel_residual=rel, allreduces=n_ar)
    rel_ref, it_ref = rel, 0  # the residual and iteration of the last replacement
    while it < max_iterations:
        for _ in range(min(chunk, max_iterations - it)):
            s_loc, qq = shard.normal_product(p)
            buf[:-1].copy_(s_loc)
            buf[-1:].copy_(qq.reshape(1))
            _allreduce(buf, group)  # the one collective of the iteration
            n_ar += 1
            pap = buf[-1]
            alpha = torch.where(pap > 0, rz / torch.where(pap > 0, pap, 1.0), zero)
            x.add_(alpha * p)
            r.sub_(alpha * buf[:-1])
            torch.mul(d, r, out=z)
            rz_new = torch.dot(r, z)
            beta = torch.where(rz != 0, rz_new / torch.where(rz != 0, rz, 1.0), zero)
            p.mul_(beta).add_(z)
            rz = rz_new
            it += 1
        if tol <= 0:
            break
        rel = rel_of(r)
        due = rel <= tol
        if shard.mixed:
            due = due or rel <= REPLACE_DROP * rel_ref or it - it_ref >= refine_every
        if due:
            # the FP64 true residual decides; it replaces the recursive one
            rt = _allreduce(shard.residual_product(x).to(torch.float64).clone(), group)
            n_ar += 1
            rel_true = rel_of(rt)
            if rel_true <= tol:
                rel = rel_true
                break
            dev = float(torch.linalg.vector_norm(r - rt))
            r.copy_(rt)
            torch.mul(d, r, out=z)
            rz = torch.dot(r, z)
            replacements += 1
            if dev > RESTART_DEVIATION * float(torch.linalg.vector_norm(rt)):
                p.copy_(z)
            rel = rel_ref = rel_true
            it_ref = it
    if tol <= 0:
        rel = rel_of(r)
    return ShardedResult(x=x, iterations=it, rel_residual=rel, allreduces=n_ar, replacements=replacements)


def split_rows(rows: int, world: int, rank: int, multiple: int = 1) -> tuple[int, int]:
    """Contiguous row range of a rank (boundaries on multiples of `multiple`)."""
    units = (rows + multiple - 1) // multiple
    lo = units * rank // world * multiple
    hi = min(rows, units * (rank + 1) // world * multiple)
    return lo, hi
