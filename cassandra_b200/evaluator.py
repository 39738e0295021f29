"""Differentiable pattern evaluator: score = A w with a hand-written adjoint.

The reference scores a position as the sum of its pattern weights
(ScoreEstimator::Eval, Pattern/Evaluator.cpp:48-54), which over a batch of
positions is the sparse product A w of the fitting path.  ``EvaluatorFunction``
wraps the device kernels as a ``torch.autograd.Function``:

* forward  ``cas_eval_forward``: score = A w over a row range (FP32);
* backward ``cas_eval_backward``: dL/dw = A' dL/dscore on the per-block
  column-sorted copy of A (deterministic, no atomics).

Minibatches are whole 16384-row blocks (``cas_block_rows``): batch membership
is fixed and the batch order is shuffled per epoch, so every batch's
transposed copy exists before training starts.  This is the Python side where
the reference's NeuralNetwork/ code trains value models.

``Trainer`` runs Adam on the Huber + L2 objective.  By default each batch's
whole step is one call of ``cas_eval_adam_step`` (three kernels: forward
with the loss and its gradient, the adjoint, and an epilogue with the L2
term and the Adam update), captured once as a CUDA graph; an epoch replays
the graphs in that epoch's shuffled order with one device-to-host read (the
epoch's loss) at its end.  ``graphs=False`` runs the same step through
autograd, ``EvaluatorFunction`` and torch.optim.Adam.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L
from .api import GroupIndexer, MatrixCSR, _ptr, _stream


def block_rows() -> int:
    return int(L.load().cas_block_rows())


def _blocks_spanned(r0: int, r1: int, br: int) -> int:
    return 0 if r1 <= r0 else (r1 + br - 1) // br - r0 // br


def _guard_graph_buffers(csr, blocks: int) -> None:
    """The library sizes its evaluator scratch for the most blocks any call
    has spanned and reallocates it when a call spans more; CUDA graphs
    captured by a Trainer hold the old buffers.  Once a Trainer captured on
    this matrix, a call over more blocks than it sized for is refused."""
    limit = getattr(csr, "_graph_blocks", None)
    if limit is not None and blocks > limit:
        raise RuntimeError(f"a call over {blocks} blocks would reallocate evaluator buffers that CUDA graphs of a "
                           f"Trainer on this matrix use (sized for {limit}); create the Trainer with the largest "
                           f"minibatch first or use graphs=False")


class EvaluatorFunction(torch.autograd.Function):
    """score = A[row0:row1] w  (A implicit 0/1, FP32)."""

    @staticmethod
    def forward(ctx, w: torch.Tensor, csr: MatrixCSR, row0: int, row1: int) -> torch.Tensor:
        if w.dtype != torch.float32 or not w.is_cuda or not w.is_contiguous():
            raise TypeError("weights must be a contiguous CUDA float32 tensor")
        if w.numel() != csr.cols():
            raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
        score = torch.empty(row1 - row0, dtype=torch.float32, device=w.device)
        L.check(L.load().cas_eval_forward(csr.handle, row0, row1, _ptr(w), _ptr(score), _stream()))
        ctx.csr, ctx.row0, ctx.row1 = csr, row0, row1
        return score

    @staticmethod
    def backward(ctx, g: torch.Tensor):
        _guard_graph_buffers(ctx.csr, _blocks_spanned(ctx.row0, ctx.row1, block_rows()))
        g = g.contiguous().to(torch.float32)
        grad = torch.empty(ctx.csr.cols(), dtype=torch.float32, device=g.device)
        L.check(L.load().cas_eval_backward(ctx.csr.handle, ctx.row0, ctx.row1, _ptr(g), _ptr(grad), _stream()))
        return grad, None, None, None


class PatternEvaluator(torch.nn.Module):
    """Pattern weights over a fixed set of positions (the training set)."""

    def __init__(self, masks, positions: torch.Tensor, mode: str = "expanded", weights: torch.Tensor | None = None):
        super().__init__()
        self.indexer = GroupIndexer(masks, mode)
        self.csr = MatrixCSR.from_positions(self.indexer, positions, "blocked")
        cols = self.indexer.index_space_size
        w = torch.zeros(cols, dtype=torch.float32, device=positions.device) if weights is None else weights
        self.weight = torch.nn.Parameter(w.to(torch.float32).contiguous())

    @property
    def rows(self) -> int:
        return self.csr.rows()

    def forward(self, row0: int = 0, row1: int | None = None) -> torch.Tensor:
        return EvaluatorFunction.apply(self.weight, self.csr, row0, self.rows if row1 is None else row1)

    def batches(self, batch: int) -> list[tuple[int, int]]:
        """Fixed block-aligned minibatches of about `batch` rows."""
        br = block_rows()
        per = max(1, batch // br) * br
        return [(r, min(r + per, self.rows)) for r in range(0, self.rows, per)]


def objective(score: torch.Tensor, target: torch.Tensor, w: torch.Tensor, delta: float, l2: float) -> torch.Tensor:
    """Mean Huber loss (delta) plus l2 * ||w||^2."""
    return torch.nn.functional.huber_loss(score, target, delta=delta) + l2 * torch.dot(w, w)


class Trainer:
    """Adam (lr; betas 0.9, 0.999; eps 1e-8) on mean Huber(delta) + l2 ||w||^2
    over the model's fixed minibatches of about `batch` rows; every epoch()
    shuffles the batch order (torch.Generator seeded with `seed`) and returns
    the mean batch loss.  graphs=True: each batch's step is one CUDA graph
    around cas_eval_adam_step (captured at construction; the weights and the
    Adam state are left as they were), replayed in the epoch's order.
    graphs=False: autograd through EvaluatorFunction and torch.optim.Adam."""

    BETAS, EPS = (0.9, 0.999), 1e-8

    def __init__(self, model: PatternEvaluator, target: torch.Tensor, batch: int = 65536, lr: float = 1e-2,
                 l2: float = 1e-4, delta: float = 4.0, seed: int = 0, graphs: bool = True):
        self.model = model
        self.target = target.to(torch.float32).contiguous()
        if self.target.numel() != model.rows:
            raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
        self.l2, self.delta = float(l2), float(delta)
        self.batches = model.batches(batch)
        self.gen = torch.Generator().manual_seed(seed)
        self.graphs = None
        w = model.weight
        if not graphs:
            self.opt = torch.optim.Adam([w], lr=lr, betas=self.BETAS, eps=self.EPS, fused=True)
            return
        br = block_rows()
        blocks = max(_blocks_spanned(r0, r1, br) for r0, r1 in self.batches)
        _guard_graph_buffers(model.csr, blocks)
        self.opts = L.AdamOpts(lr, self.BETAS[0], self.BETAS[1], self.EPS, self.l2, self.delta)
        self._m = torch.zeros_like(w.detach())
        self._v = torch.zeros_like(w.detach())
        self._step_count = torch.zeros((), dtype=torch.int64, device=w.device)
        self._loss_sum = torch.zeros((), dtype=torch.float64, device=w.device)
        # one step outside the capture (it sizes the library's buffers for
        # the largest batch), then the state as it was before it
        w0 = w.detach().clone()
        big = max(range(len(self.batches)), key=lambda i: self.batches[i][1] - self.batches[i][0])
        self._step(big)
        torch.cuda.synchronize(w.device)
        with torch.no_grad():
            w.copy_(w0)
        for t in (self._m, self._v, self._step_count, self._loss_sum):
            t.zero_()
        pool = torch.cuda.graph_pool_handle()
        self.graphs = []
        for i in range(len(self.batches)):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, pool=pool):
                self._step(i)
            self.graphs.append(g)
        model.csr._graph_blocks = max(getattr(model.csr, "_graph_blocks", None) or 0, blocks)

    def _step(self, i: int):
        r0, r1 = self.batches[i]
        w = self.model.weight
        L.check(L.load().cas_eval_adam_step(self.model.csr.handle, r0, r1, _ptr(self.target[r0:r1]), _ptr(w),
                                            _ptr(self._m), _ptr(self._v), _ptr(self._step_count),
                                            _ptr(self._loss_sum), C.byref(self.opts), _stream()))

    def epoch(self) -> float:
        order = torch.randperm(len(self.batches), generator=self.gen).tolist()
        if self.graphs is not None:
            self._loss_sum.zero_()
            for i in order:
                self.graphs[i].replay()
            return float(self._loss_sum) / len(self.batches)
        model, total = self.model, torch.zeros((), dtype=torch.float32, device=self.model.weight.device)
        for i in order:
            r0, r1 = self.batches[i]
            self.opt.zero_grad(set_to_none=True)
            loss = objective(model(r0, r1), self.target[r0:r1], model.weight, self.delta, self.l2)
            loss.backward()
            self.opt.step()
            total += loss.detach()
        return float(total) / len(self.batches)


def train(model: PatternEvaluator, target: torch.Tensor, epochs: int = 5, batch: int = 65536, lr: float = 1e-2,
          l2: float = 1e-4, delta: float = 4.0, seed: int = 0, graphs: bool = True) -> list[float]:
    """Adam on the Huber + L2 objective over fixed minibatches whose order is
    shuffled every epoch.  Returns the mean batch loss of every epoch."""
    t = Trainer(model, target, batch=batch, lr=lr, l2=l2, delta=delta, seed=seed, graphs=graphs)
    return [t.epoch() for _ in range(epochs)]


def full_objective(model: PatternEvaluator, target: torch.Tensor, w: torch.Tensor | None = None,
                   delta: float = 4.0, l2: float = 1e-4) -> float:
    """The objective over all rows for weights w (default: the model's)."""
    w = model.weight.detach() if w is None else w.to(torch.float32).contiguous()
    with torch.no_grad():
        s = EvaluatorFunction.apply(w, model.csr, 0, model.rows)
        return float(objective(s, target.to(torch.float32), w, delta, l2))


def central_difference(model: PatternEvaluator, target: torch.Tensor, coords: torch.Tensor, row0: int, row1: int,
                       h: float = 0.25) -> torch.Tensor:
    """Central finite differences of L(w) = 0.5 ||A w - t||^2 over [row0, row1)
    (evaluated in FP64 from the FP32 scores) at the given coordinates."""
    w = model.weight.detach().clone()
    t = target[row0:row1].to(torch.float64)
    out = torch.empty(len(coords), dtype=torch.float64)
    for j, c in enumerate(coords.tolist()):
        vals = []
        for sgn in (1.0, -1.0):
            wp = w.clone()
            wp[c] += sgn * h
            s = EvaluatorFunction.apply(wp, model.csr, row0, row1).to(torch.float64)
            vals.append(0.5 * float(torch.sum((s - t) ** 2)))
        out[j] = (vals[0] - vals[1]) / (2 * h)
    return out


__all__ = ["EvaluatorFunction", "PatternEvaluator", "Trainer", "train", "objective", "full_objective",
           "central_difference", "block_rows"]
