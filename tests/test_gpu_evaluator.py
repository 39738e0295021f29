"""The differentiable evaluator: forward A w and the hand-written adjoint
A' g behind torch.autograd.Function, against the oracle, the compiled
reference's x * A, central finite differences, and a short training run."""
import ctypes as C

import numpy as np
import pytest
import torch

import cassandra_b200 as cb
from cassandra_b200 import evaluator as ev
from tests.golden.make_golden import SET8

pytestmark = pytest.mark.gpu

BR = 16384


@pytest.fixture(scope="module")
def setup(orc):
    rows = 3 * BR + 1234  # three full blocks and a partial one
    pos = cb.generate_positions(44, rows, 10, 50)
    model = ev.PatternEvaluator(SET8, pos, "expanded")
    idx = orc.group_index(SET8, 1, pos.cpu().numpy().view(np.uint64))
    rng = np.random.default_rng(44)
    w = rng.normal(0, 0.5, model.weight.numel()).astype(np.float32)
    with torch.no_grad():
        model.weight.copy_(torch.from_numpy(w))
    target = torch.from_numpy(np.clip(2 * np.rint(orc.spmv(idx, len(w), w.astype(np.float64)) / 2), -64, 64)
                              .astype(np.float32)).cuda()
    return model, idx, w, target


def test_block_rows():
    assert ev.block_rows() == BR


@pytest.mark.parametrize("r0,r1", [(0, BR), (BR, 3 * BR), (3 * BR, 3 * BR + 1234), (0, 3 * BR + 1234), (5, 77)])
def test_forward_matches_oracle(cuda, orc, setup, r0, r1):
    model, idx, w, _ = setup
    got = model(r0, r1).detach().cpu().numpy().astype(np.float64)
    want = orc.spmv(idx[r0:r1], len(w), w.astype(np.float64))
    assert np.abs(got - want).max() <= 64 * 2 ** -23 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("r0,r1", [(0, BR), (BR, 3 * BR), (3 * BR, 3 * BR + 1234), (0, 3 * BR + 1234)])
def test_adjoint_matches_oracle_and_reference(cuda, orc, setup, r0, r1):
    model, idx, w, _ = setup
    g = torch.randn(r1 - r0, dtype=torch.float32, device="cuda")
    s = model(r0, r1)
    (grad,) = torch.autograd.grad(s, model.weight, g)
    gh = g.cpu().numpy()
    want = orc.spmv_t(idx[r0:r1], len(w), gh.astype(np.float64))
    scale = np.abs(want).max()
    np.testing.assert_allclose(grad.cpu().numpy(), want, rtol=0, atol=1e-5 * scale)
    import oracle

    if oracle.ref_available():
        sub = np.ascontiguousarray(idx[r0:r1])
        ref = np.empty(len(w), np.float32)
        oracle.ref_lib().ref_spmv_t(sub.shape[1], sub.shape[0], len(w), sub.ctypes.data_as(C.c_void_p),
                                    gh.ctypes.data_as(C.c_void_p), ref.ctypes.data_as(C.c_void_p))
        np.testing.assert_allclose(grad.cpu().numpy(), ref, rtol=0, atol=2e-5 * scale)
    # deterministic: the same bits twice
    (grad2,) = torch.autograd.grad(model(r0, r1), model.weight, g)
    assert grad.cpu().numpy().tobytes() == grad2.cpu().numpy().tobytes()


def test_adjoint_rejects_unaligned_ranges(cuda, setup):
    model, _, _, _ = setup
    s = model(5, BR)
    with pytest.raises(cb.CasError):
        s.sum().backward()


def test_gradient_matches_central_differences(cuda, setup):
    model, idx, w, target = setup
    r0, r1 = BR, 2 * BR
    s = model(r0, r1)
    loss = 0.5 * torch.sum((s.double() - target[r0:r1].double()) ** 2)
    (grad,) = torch.autograd.grad(loss, model.weight)
    rng = np.random.default_rng(1)
    hit = np.unique(idx[r0:r1])
    coords = np.concatenate([rng.choice(hit, 900, replace=False),
                             rng.choice(np.setdiff1d(np.arange(len(w)), hit), 100, replace=False)])
    fd = ev.central_difference(model, target, torch.from_numpy(coords), r0, r1).numpy()
    got = grad.detach().cpu().numpy()[coords].astype(np.float64)
    np.testing.assert_allclose(got, fd, rtol=1e-3, atol=1e-2)


def test_training_reduces_loss_towards_least_squares(cuda, orc, setup):
    rows = 6 * BR
    pos = cb.generate_positions(45, rows, 10, 50)
    model = ev.PatternEvaluator(SET8, pos, "expanded")
    g = cb.GroupIndexer(SET8, "expanded")
    a = cb.MatrixCSR.from_positions(g, pos, "rows")
    b = cb.generate_targets(a, 45)
    target = b.float()
    before = ev.full_objective(model, target)
    hist = ev.train(model, target, epochs=5, batch=2 * BR, lr=1e-2, l2=1e-4, delta=4.0, seed=0)
    after = ev.full_objective(model, target)
    assert hist[-1] < hist[0] and after < before
    s = cb.PCG(a, b, tol=1e-8)
    assert s.run()["converged"]
    ls_obj = ev.full_objective(model, target, s.x().float())
    # Adam on Huber+L2 for 5 epochs lands in the same range as the
    # least-squares optimum evaluated on the same objective
    assert after <= 3.0 * ls_obj + 1.0, (after, ls_obj)


def test_graph_trainer_matches_autograd(cuda):
    """The CUDA-graph training step (manual loss gradient, the same kernels,
    fused Adam) follows the autograd step through EvaluatorFunction, batch
    order included; a ragged last batch (a partial block) is part of it."""
    rows = 6 * BR + 1000
    pos = cb.generate_positions(46, rows, 10, 50)
    g = cb.GroupIndexer(SET8, "expanded")
    target = cb.generate_targets(cb.MatrixCSR.from_positions(g, pos, "rows"), 46).float()
    m_auto = ev.PatternEvaluator(SET8, pos, "expanded")
    m_graph = ev.PatternEvaluator(SET8, pos, "expanded")
    h_auto = ev.train(m_auto, target, epochs=3, batch=2 * BR, seed=3, graphs=False)
    t = ev.Trainer(m_graph, target, batch=2 * BR, seed=3)
    assert len(t.graphs) == len(t.batches) == 4
    assert torch.count_nonzero(m_graph.weight) == 0  # capture changed nothing
    h_graph = [t.epoch() for _ in range(3)]
    np.testing.assert_allclose(h_graph, h_auto, rtol=1e-4)
    torch.testing.assert_close(m_graph.weight.detach(), m_auto.weight.detach(), rtol=1e-3, atol=1e-4)
    assert h_graph[-1] < h_graph[0]


def test_fused_adam_step_matches_torch(cuda, setup):
    """cas_eval_adam_step on one minibatch (the partial last block included)
    against the same step written in torch: the objective's value, its
    gradient through the adjoint, and Adam's update of w, m, v."""
    from cassandra_b200 import _lib as L

    model, _, w0, target = setup
    r0, r1 = 2 * BR, model.rows
    w = torch.from_numpy(w0).cuda()
    m = torch.full_like(w, 0.01)
    v = torch.full_like(w, 0.02)
    step = torch.tensor(4, dtype=torch.int64, device="cuda")
    loss = torch.tensor(1.5, dtype=torch.float64, device="cuda")
    lr, b1, b2, eps, l2, delta = 1e-2, 0.9, 0.999, 1e-8, 1e-4, 4.0
    # the reference step in torch, from the same state
    t = target[r0:r1]
    score = ev.EvaluatorFunction.apply(w, model.csr, r0, r1)
    want_loss = float(ev.objective(score, t, w, delta, l2))
    ds = (score - t).clamp(-delta, delta) / (r1 - r0)
    g = torch.empty_like(w)
    L.check(L.load().cas_eval_backward(model.csr.handle, r0, r1, ds.data_ptr(), g.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream))
    g = g + 2 * l2 * w
    m_want = m + (1 - b1) * (g - m)
    v_want = b2 * v + (1 - b2) * g * g
    k = 5
    w_want = w - lr / (1 - b1 ** k) * m_want / (v_want.sqrt() / (1 - b2 ** k) ** 0.5 + eps)
    opts = L.AdamOpts(lr, b1, b2, eps, l2, delta)
    L.check(L.load().cas_eval_adam_step(model.csr.handle, r0, r1, t.data_ptr(), w.data_ptr(), m.data_ptr(),
                                        v.data_ptr(), step.data_ptr(), loss.data_ptr(), C.byref(opts),
                                        torch.cuda.current_stream().cuda_stream))
    assert int(step) == k
    assert float(loss) == pytest.approx(1.5 + want_loss, rel=1e-5)
    torch.testing.assert_close(m, m_want, rtol=1e-5, atol=1e-8)
    torch.testing.assert_close(v, v_want, rtol=1e-5, atol=1e-10)
    torch.testing.assert_close(w, w_want, rtol=1e-5, atol=1e-6)
    with pytest.raises(cb.CasError):  # an unaligned minibatch is refused
        L.check(L.load().cas_eval_adam_step(model.csr.handle, 1, BR, t.data_ptr(), w.data_ptr(), m.data_ptr(),
                                            v.data_ptr(), step.data_ptr(), loss.data_ptr(), C.byref(opts),
                                            torch.cuda.current_stream().cuda_stream))


def test_graph_trainer_guards_its_buffers(cuda):
    """After a Trainer captured its graphs for one-block minibatches, calls
    that would grow (and so reallocate) the matrix's evaluator scratch are
    refused; calls within the captured size still run."""
    rows = 4 * BR
    pos = cb.generate_positions(47, rows, 10, 50)
    model = ev.PatternEvaluator(SET8, pos, "expanded")
    target = torch.zeros(rows, dtype=torch.float32, device="cuda")
    ev.Trainer(model, target, batch=BR)
    with pytest.raises(RuntimeError, match="reallocate"):
        ev.Trainer(model, target, batch=2 * BR)
    with pytest.raises(RuntimeError, match="reallocate"):
        model(0, rows).sum().backward()
    assert np.isfinite(ev.Trainer(model, target, batch=BR, graphs=False).epoch())


def test_captured_scratch_never_moves(cuda):
    """The rule behind the graph trainer, enforced in the library itself
    (direct C calls, no Python guard): once a training step has been
    captured into a CUDA graph, a call that would grow (and so free) the
    matrix's evaluator scratch is refused, eager or captured; growing it
    during a capture is refused too; calls within the size run and the
    captured graph still replays."""
    from cassandra_b200 import _lib as L

    lib = L.load()
    rows = 3 * BR
    pos = cb.generate_positions(48, rows, 10, 50)
    opts = L.AdamOpts(1e-2, 0.9, 0.999, 1e-8, 1e-4, 4.0)

    def state(cols):
        return [torch.zeros(cols, dtype=torch.float32, device="cuda") for _ in range(3)] + \
               [torch.zeros((), dtype=torch.int64, device="cuda"), torch.zeros((), dtype=torch.float64, device="cuda")]

    def step(model, r0, r1, st, target):
        w, m, v, n, loss = st
        return lib.cas_eval_adam_step(model.csr.handle, r0, r1, target.data_ptr(), w.data_ptr(), m.data_ptr(),
                                      v.data_ptr(), n.data_ptr(), loss.data_ptr(), C.byref(opts),
                                      torch.cuda.current_stream().cuda_stream)

    model = ev.PatternEvaluator(SET8, pos, "expanded")
    target = torch.ones(rows, dtype=torch.float32, device="cuda")
    st = state(model.weight.numel())
    L.check(step(model, 0, BR, st, target))  # sizes the scratch for one block
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            L.check(step(model, BR, 2 * BR, st, target))
    torch.cuda.current_stream().wait_stream(s)
    assert step(model, 0, 2 * BR, st, target) == L.CAS_ERR_INVALID_ARGUMENT
    assert "captured" in L.last_error()
    L.check(step(model, 2 * BR, 3 * BR, st, target))
    g.replay()
    torch.cuda.synchronize()
    assert int(st[3]) == 3 and np.isfinite(float(st[4]))

    fresh = ev.PatternEvaluator(SET8, pos, "expanded")
    st2 = state(fresh.weight.numel())
    g2 = torch.cuda.CUDAGraph()
    with pytest.raises(cb.CasError, match="before capturing"):
        with torch.cuda.graph(g2):
            L.check(step(fresh, 0, BR, st2, target))
