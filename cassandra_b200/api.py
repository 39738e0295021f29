"""Python mirror of the reference's fitting API over the C ABI.

Names follow the reference: ``GroupIndexer`` (Pattern/Indexer.h:29-40),
``MatrixCSR`` with ``A @ x`` / ``x @ A`` (Math/MatrixCSR.h:11-33),
``jacobi_preconditioner_of_ata`` (Math/MatrixCSR.h:30), the iterative solvers
``PCG``, ``CG``, ``LSQR`` and ``LSMR`` with ``iterate`` / ``residuum`` / ``x`` / ``error``
(Math/Solver.h:9-287), and ``fit_weights`` (PatternFit/PatternFit.cpp:7-39).

Device data is exchanged as CUDA torch tensors (PyTorch is used only for
device memory and the current stream); host data as numpy arrays.  Size
errors raise ``SizeMismatch`` like the reference's ``runtime_error("Size
mismatch.")``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L

_REF_MODES = {"reference": L.CAS_INDEX_REFERENCE, "expanded": L.CAS_INDEX_EXPANDED}


def _stream() -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor | None) -> C.c_void_p:
    return C.c_void_p(t.data_ptr() if t is not None else 0)


def _sync_before_free() -> None:
    """Waits for the current stream before a handle's device memory goes back.
    At interpreter exit the torch module may already be torn down; nothing
    is left to wait for then."""
    try:
        cuda = torch.cuda
        if cuda.is_initialized():
            cuda.current_stream().synchronize()
    except (AttributeError, TypeError):  # module attributes already cleared
        pass


def _require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


class GroupIndexer:
    """GroupIndexer(std::vector<uint64_t>) (Pattern/Indexer.cpp:382-392).

    mode="reference" is bit-exact with the reference; mode="expanded" uses
    3^k columns and all 8 symmetry instances for every mask."""

    def __init__(self, masks, mode: str = "reference"):
        self._lib = L.load()
        m = np.ascontiguousarray(masks, dtype=np.uint64)
        if m.ndim != 1 or len(m) == 0:
            raise ValueError("masks must be a non-empty 1-D sequence")
        self.masks = m
        self.mode = mode
        h = C.c_void_p()
        L.check(self._lib.cas_patterns_create(m.ctypes.data_as(C.c_void_p), len(m), _REF_MODES[mode], C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.cas_patterns_destroy(h)
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def index_space_size(self) -> int:
        return int(self._lib.cas_patterns_cols(self._h))

    @property
    def nnz_per_row(self) -> int:
        return int(self._lib.cas_patterns_nnz_per_row(self._h))

    def variations(self) -> np.ndarray:
        out = np.empty(self.nnz_per_row, dtype=np.uint64)
        L.check(self._lib.cas_patterns_variations(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def indexer(self, i: int) -> dict:
        sp, order, space, off = C.c_uint64(), C.c_int(), C.c_int64(), C.c_int64()
        L.check(self._lib.cas_patterns_indexer(self._h, i, C.byref(sp), C.byref(order), C.byref(space),
                                               C.byref(off)))
        return {"pattern": sp.value, "order": order.value, "space": space.value, "offset": off.value}

    def indices(self, positions: torch.Tensor) -> torch.Tensor:
        """positions: CUDA int64 [n, 2] (P, O) -> int32 [n, K] (uint32 bit patterns)."""
        _require_cuda(positions, "positions")
        n = positions.shape[0]
        out = torch.empty((n, self.nnz_per_row), dtype=torch.int32, device=positions.device)
        L.check(self._lib.cas_index(self._h, _ptr(positions), n, _ptr(out), _stream()))
        return out


class MatrixCSR:
    """Device-resident MatrixCSR with implicit 1.0 entries and its transposed copy."""

    def __init__(self, handle: C.c_void_p, keep=None):
        self._lib = L.load()
        self._h = handle
        self._keep = keep

    @classmethod
    def from_positions(cls, indexer: GroupIndexer, positions: torch.Tensor, layouts: str | None = None) -> "MatrixCSR":
        """layouts: None (both where possible), "rows", "blocked" or "rows+blocked"."""
        _require_cuda(positions, "positions")
        lib = L.load()
        h = C.c_void_p()
        if layouts is None:
            L.check(lib.cas_csr_from_positions(indexer.handle, _ptr(positions), positions.shape[0], _stream(),
                                               C.byref(h)))
        else:
            mask = sum({"rows": L.CAS_LAYOUT_ROWS, "blocked": L.CAS_LAYOUT_BLOCKED}[x] for x in layouts.split("+"))
            L.check(lib.cas_csr_from_positions_layout(indexer.handle, _ptr(positions), positions.shape[0], mask,
                                                      _stream(), C.byref(h)))
        return cls(h, keep=indexer)

    @classmethod
    def from_positions_batched(cls, indexer: GroupIndexer, positions: torch.Tensor,
                               problem_rows) -> "MatrixCSR":
        """A batch of independent fits over the same patterns (one per
        empty-count stage): problem q is the next problem_rows[q] positions
        and owns columns [q * C, (q + 1) * C).  The result is the
        block-diagonal matrix of the problems, in the blocked layout."""
        _require_cuda(positions, "positions")
        lib = L.load()
        rows = np.ascontiguousarray(np.asarray(problem_rows, dtype=np.int64))
        if int(rows.sum()) != positions.shape[0]:
            raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
        h = C.c_void_p()
        L.check(lib.cas_csr_from_positions_batched(indexer.handle, _ptr(positions), rows.ctypes.data_as(C.c_void_p),
                                                   len(rows), _stream(), C.byref(h)))
        return cls(h, keep=indexer)

    def problems(self) -> np.ndarray:
        """First row of every problem and the total (problems + 1 entries)."""
        n = int(self._lib.cas_csr_problems(self._h, None))
        out = np.zeros(n + 1, dtype=np.int64)
        self._lib.cas_csr_problems(self._h, out.ctypes.data_as(C.c_void_p))
        return out

    def schedules(self) -> dict:
        """A'y schedules timed by the build-time autotuner on this matrix and
        the one in use (blocked layout only)."""
        out = (L.Schedule * 16)()
        cur = L.Schedule()
        n = self._lib.cas_csr_schedules(self.handle, out, 16, C.byref(cur))
        if n < 0:
            return {}
        return {"in_use": cur.as_dict(), "timed": [out[i].as_dict() for i in range(n)]}

    def layouts(self) -> set[str]:
        m = int(self._lib.cas_csr_layouts(self._h))
        return {n for n, bit in (("rows", L.CAS_LAYOUT_ROWS), ("blocked", L.CAS_LAYOUT_BLOCKED)) if m & bit}

    @classmethod
    def from_indices(cls, indices: torch.Tensor, cols: int) -> "MatrixCSR":
        """indices: CUDA int32 [rows, K] (column indices, copied)."""
        _require_cuda(indices, "indices")
        lib = L.load()
        h = C.c_void_p()
        L.check(lib.cas_csr_from_indices(_ptr(indices), indices.shape[1], indices.shape[0], cols, _stream(),
                                         C.byref(h)))
        return cls(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _sync_before_free()
            self._lib.cas_csr_destroy(h)
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def rows(self) -> int:
        return int(self._lib.cas_csr_rows(self._h))

    def cols(self) -> int:
        return int(self._lib.cas_csr_cols(self._h))

    @property
    def nnz_per_row(self) -> int:
        return int(self._lib.cas_csr_nnz_per_row(self._h))

    def indices(self) -> torch.Tensor:
        """Copy of the row-major column indices (int32 [rows, K])."""
        src = self._lib.cas_csr_indices(self._h)
        if not src and self.rows() > 0:
            raise ValueError("this CSR has no rows layout (built with layouts='blocked')")
        return _device_view(src, (self.rows(), self.nnz_per_row), "<i4").clone()

    def transposed(self) -> tuple[torch.Tensor, torch.Tensor]:
        """Copies of (col_ptr int64 [cols+1], row_idx int32 [nnz]) of the transposed copy."""
        cp, ri = C.c_void_p(), C.c_void_p()
        L.check(self._lib.cas_csr_transposed(self._h, C.byref(cp), C.byref(ri)))
        if not cp.value:
            raise ValueError("this CSR has no rows layout (built with layouts='blocked')")
        col_ptr = _device_view(cp.value, (self.cols() + 1,), "<i8").clone()
        row_idx = _device_view(ri.value, (self.rows() * self.nnz_per_row,), "<i4").clone()
        return col_ptr, row_idx

    def _dtype(self, t: torch.Tensor) -> int:
        if t.dtype == torch.float32:
            return L.CAS_F32
        if t.dtype == torch.float64:
            return L.CAS_F64
        raise TypeError("vectors must be float32 or float64")

    def matvec(self, x: torch.Tensor) -> torch.Tensor:
        """A x (operator*(const MatrixCSR&, const Vector&))."""
        _require_cuda(x, "x")
        if x.numel() != self.cols():
            raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
        y = torch.empty(self.rows(), dtype=x.dtype, device=x.device)
        L.check(self._lib.cas_spmv(self._h, self._dtype(x), _ptr(x), _ptr(y), _stream()))
        return y

    def rmatvec(self, y: torch.Tensor) -> torch.Tensor:
        """A' y, i.e. the reference's y * A (operator*(const Vector&, const MatrixCSR&))."""
        _require_cuda(y, "y")
        if y.numel() != self.rows():
            raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
        x = torch.empty(self.cols(), dtype=y.dtype, device=y.device)
        L.check(self._lib.cas_spmv_t(self._h, self._dtype(y), _ptr(y), _ptr(x), _stream()))
        return x

    def __matmul__(self, x: torch.Tensor) -> torch.Tensor:
        return self.matvec(x)

    def __rmatmul__(self, y: torch.Tensor) -> torch.Tensor:
        return self.rmatvec(y)


class _CudaArray:
    """Borrowed view of library-owned device memory (CUDA array interface v3)."""

    def __init__(self, ptr: int, shape: tuple, typestr: str):
        self.__cuda_array_interface__ = {"data": (int(ptr or 0), False), "shape": tuple(shape), "typestr": typestr,
                                         "version": 3, "strides": None}


def _device_view(ptr: int, shape: tuple, typestr: str) -> torch.Tensor:
    if int(np.prod(shape)) == 0:
        return torch.empty(shape, dtype={"<i4": torch.int32, "<i8": torch.int64}[typestr], device="cuda")
    return torch.as_tensor(_CudaArray(ptr, shape, typestr), device="cuda")


def jacobi_preconditioner_of_ata(a: MatrixCSR, dtype=torch.float64) -> torch.Tensor:
    """1 / diag(A'A) (Math/MatrixCSR.cpp:21-47); empty columns give inf."""
    out = torch.empty(a.cols(), dtype=dtype, device="cuda")
    L.check(a._lib.cas_jacobi(a.handle, L.CAS_F32 if dtype == torch.float32 else L.CAS_F64, _ptr(out), _stream()))
    return out


def solve_opts(method: str = "pcg", precision: str = "fp64", tol: float = 1e-8, max_iterations: int = 20000,
               refine_every: int = 50, check_every: int = 50, jacobi: bool = True,
               scale_columns: bool = False) -> L.SolveOpts:
    """cas_solve_opts.  scale_columns: LSQR/LSMR iterate on A S with S =
    diag(A'A)^-1/2 (the reference's LSQR/LSMR are unscaled: False)."""
    o = L.SolveOpts()
    L.load().cas_solve_opts_default(C.byref(o))
    o.method = {"pcg": L.CAS_PCG, "lsqr": L.CAS_LSQR, "cg": L.CAS_CG, "lsmr": L.CAS_LSMR}[method]
    o.precision = {"fp64": L.CAS_PLAIN_FP64, "mixed": L.CAS_MIXED}[precision]
    o.tol = tol
    o.max_iterations = max_iterations
    o.refine_every = refine_every
    o.check_every = check_every
    o.jacobi = int(jacobi)
    o.scale_columns = int(scale_columns)
    return o


class _Solver:
    """IterativeSolver (Math/Solver.h:9-16) over a device-resident system."""

    method = "pcg"

    def __init__(self, a: MatrixCSR, b: torch.Tensor, x0: torch.Tensor | None = None, precision: str = "fp64",
                 tol: float = 0.0, max_iterations: int = 1 << 30, refine_every: int = 50, check_every: int = 50,
                 jacobi: bool = True, scale_columns: bool = False):
        _require_cuda(b, "b")
        if b.dtype != torch.float64:
            b = b.double()
        if b.numel() != a.rows():
            raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
        if x0 is not None:
            x0 = x0.double().contiguous()
            if x0.numel() != a.cols():
                raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
        self._lib = L.load()
        self.a = a
        self.b = b.contiguous()
        self.opts = solve_opts(self.method, precision, tol, max_iterations, refine_every, check_every, jacobi,
                               scale_columns)
        h = C.c_void_p()
        L.check(self._lib.cas_solver_create(a.handle, C.byref(self.opts), _ptr(self.b), _ptr(x0), _stream(),
                                            C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.cas_solver_destroy(h)
            self._h = None

    def iterate(self, n: int = 1) -> None:
        L.check(self._lib.cas_solver_iterate(self._h, n))

    def residuum(self) -> float:
        v = C.c_double()
        L.check(self._lib.cas_solver_residuum(self._h, C.byref(v)))
        return v.value

    def x(self) -> torch.Tensor:
        out = torch.empty(self.a.cols(), dtype=torch.float64, device="cuda")
        L.check(self._lib.cas_solver_x(self._h, _ptr(out)))
        return out

    def rel_residual(self) -> float:
        v = C.c_double()
        L.check(self._lib.cas_solver_rel_residual(self._h, C.byref(v)))
        return v.value

    def iterations(self) -> int:
        return int(self._lib.cas_solver_iterations(self._h))

    def save_state(self) -> np.ndarray:
        """The solver's state as a host byte array (cas_solver_save_state):
        a checkpoint that load_state() resumes from."""
        n = C.c_size_t()
        L.check(self._lib.cas_solver_state_size(self._h, C.byref(n)))
        buf = np.empty(n.value, dtype=np.uint8)
        L.check(self._lib.cas_solver_save_state(self._h, buf.ctypes.data_as(C.c_void_p), n.value))
        return buf

    def load_state(self, state) -> None:
        """Resumes from a checkpoint of save_state() (same method, precision,
        column scaling, matrix and right-hand side)."""
        buf = np.ascontiguousarray(np.frombuffer(state, dtype=np.uint8) if isinstance(state, (bytes, bytearray))
                                   else state, dtype=np.uint8)
        L.check(self._lib.cas_solver_load_state(self._h, buf.ctypes.data_as(C.c_void_p), buf.nbytes))

    def run(self) -> dict:
        rep = L.SolveReport()
        st = self._lib.cas_solver_run(self._h, C.byref(rep))
        if st not in (L.CAS_OK, L.CAS_ERR_NOT_CONVERGED):
            L.check(st)
        d = rep.as_dict()
        d["converged"] = st == L.CAS_OK
        return d


class PCG(_Solver):
    """PCG(transposed(A) * A, DiagonalPreconditioner(Jacobi), x0, transposed(A) * b)."""

    method = "pcg"


class CG(_Solver):
    """CG on A'A x = A'b (Math/Solver.h:40-76)."""

    method = "cg"


class LSQR(_Solver):
    """LSQR(A, x0, b) (Math/Solver.h:128-182).  scale_columns=True iterates
    on A S, S = diag(A'A)^-1/2, and returns x = S y (not in the reference)."""

    method = "lsqr"


class LSMR(_Solver):
    """LSMR(A, x0, b) (Math/Solver.h:222-287).  residuum() is 0, as the
    reference's Residuum(); rel_residual() is the FP64 true one."""

    method = "lsmr"


def solve_batched(a: MatrixCSR, b: torch.Tensor, precision: str = "mixed", tol: float = 1e-8,
                  max_iterations: int = 20000, refine_every: int = 50, check_every: int = 50, method: str = "pcg",
                  jacobi: bool = True) -> tuple[torch.Tensor, list[dict], bool]:
    """Every problem of a batched matrix solved by its own PCG (or CG) in one
    run (cas_solve_batched).  Returns x as [problems, C], one report per
    problem and whether all reached the tolerance."""
    _require_cuda(b, "b")
    b = b.double().contiguous()
    if b.numel() != a.rows():
        raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
    lib = L.load()
    n = len(a.problems()) - 1
    opts = solve_opts(method, precision, tol, max_iterations, refine_every, check_every, jacobi)
    x = torch.empty(a.cols(), dtype=torch.float64, device="cuda")
    reps = (L.SolveReport * n)()
    st = lib.cas_solve_batched(a.handle, C.byref(opts), _ptr(b), _ptr(x), reps, _stream())
    if st not in (L.CAS_OK, L.CAS_ERR_NOT_CONVERGED):
        L.check(st)
    out = []
    for r in reps:
        d = r.as_dict()
        d["converged"] = bool(tol <= 0 or d["rel_residual"] <= tol)
        out.append(d)
    return x.view(n, -1), out, st == L.CAS_OK


def fit_weights_batched(indexer: GroupIndexer, positions: torch.Tensor, scores: torch.Tensor, sizes,
                        method: str = "pcg", precision: str = "mixed", tol: float = 1e-8,
                        max_iterations: int = 20000, refine_every: int = 50, check_every: int = 50,
                        jacobi: bool = True, scale_columns: bool = False) -> tuple[torch.Tensor, list[dict], bool]:
    """The per-stage fits of the training loop in one call
    (cas_fit_weights_batched_device): problem q is the next sizes[q]
    positions (device {P, O} int64 pairs) and scores.  PCG/CG run as one
    batched solve on a block-diagonal layout; LSQR/LSMR as one solver per
    problem, all run together.  Returns the weights as [problems, cols], one
    report per problem and whether all reached the tolerance."""
    _require_cuda(positions, "positions")
    _require_cuda(scores, "scores")
    sizes = np.ascontiguousarray(sizes, dtype=np.int64)
    if positions.shape[0] != int(sizes.sum()) or scores.numel() != int(sizes.sum()):
        raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
    pos = positions.contiguous()
    sc = scores.double().contiguous()
    lib = L.load()
    n = len(sizes)
    opts = solve_opts(method, precision, tol, max_iterations, refine_every, check_every, jacobi, scale_columns)
    x = torch.empty(n * indexer.index_space_size, dtype=torch.float64, device="cuda")
    reps = (L.SolveReport * n)()
    st = lib.cas_fit_weights_batched_device(indexer.handle, _ptr(pos), _ptr(sc),
                                            sizes.ctypes.data_as(C.c_void_p), n, C.byref(opts), _ptr(x), reps,
                                            _stream())
    if st not in (L.CAS_OK, L.CAS_ERR_NOT_CONVERGED):
        L.check(st)
    out = []
    for r in reps:
        d = r.as_dict()
        d["converged"] = bool(tol <= 0 or d["rel_residual"] <= tol)
        out.append(d)
    return x.view(n, -1), out, st == L.CAS_OK


def fit_weights(masks, positions: np.ndarray, scores: np.ndarray, mode: str = "reference", method: str = "pcg",
                precision: str = "fp64", tol: float = 1e-8, max_iterations: int = 20000,
                refine_every: int = 50, check_every: int = 50, scale_columns: bool = False) -> tuple[np.ndarray, dict]:
    """FitWeights with host buffers in and out (PatternFit/PatternFit.cpp:7-39).

    tol <= 0 runs exactly max_iterations iterations, as the reference's
    FitWeights(pattern, positions, iterations) does."""
    lib = L.load()
    m = np.ascontiguousarray(masks, dtype=np.uint64)
    pos = np.ascontiguousarray(positions, dtype=np.uint64).reshape(-1, 2)
    sc = np.ascontiguousarray(scores, dtype=np.float32)
    if len(sc) != len(pos):
        raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
    h = C.c_void_p()
    L.check(lib.cas_patterns_create(m.ctypes.data_as(C.c_void_p), len(m), _REF_MODES[mode], C.byref(h)))
    cols = int(lib.cas_patterns_cols(h))
    lib.cas_patterns_destroy(h)
    w = np.empty(cols, dtype=np.float32)
    o = solve_opts(method, precision, tol, max_iterations, refine_every, check_every, scale_columns=scale_columns)
    rep = L.SolveReport()
    st = lib.cas_fit_weights(m.ctypes.data_as(C.c_void_p), len(m), _REF_MODES[mode], pos.ctypes.data_as(C.c_void_p),
                             sc.ctypes.data_as(C.c_void_p), len(pos), C.byref(o), w.ctypes.data_as(C.c_void_p),
                             C.byref(rep))
    if st not in (L.CAS_OK, L.CAS_ERR_NOT_CONVERGED):
        L.check(st)
    d = rep.as_dict()
    d["converged"] = st == L.CAS_OK
    return w, d


def generate_positions(seed: int, n: int, min_empties: int, max_empties: int, device="cuda") -> torch.Tensor:
    """Seeded random-play positions as CUDA int64 [n, 2]."""
    out = torch.empty((n, 2), dtype=torch.int64, device=device)
    L.check(L.load().cas_generate_positions(seed, n, min_empties, max_empties, _ptr(out), _stream()))
    return out


def generate_positions_host(seed: int, first: int, n: int, min_empties: int, max_empties: int) -> np.ndarray:
    out = np.empty((n, 2), dtype=np.uint64)
    L.check(L.load().cas_generate_positions_host(seed, first, n, min_empties, max_empties,
                                                 out.ctypes.data_as(C.c_void_p)))
    return out


def generate_targets(a: MatrixCSR, seed: int, w_sigma: float = 0.5, noise_sigma: float = 4.0,
                     return_true_weights: bool = False, first_row: int = 0):
    """Seeded targets b = clamp(2 rint((A w* + e) / 2), -64, 64); the rows of
    `a` are rows first_row.. of the whole system (a rank's block)."""
    b = torch.empty(a.rows(), dtype=torch.float64, device="cuda")
    w = torch.empty(a.cols(), dtype=torch.float64, device="cuda") if return_true_weights else None
    L.check(L.load().cas_generate_targets_rows(a.handle, seed, w_sigma, noise_sigma, first_row, _ptr(b), _ptr(w),
                                               _stream()))
    return (b, w) if return_true_weights else b


# ---------------------------------------------------------------------------
# Pattern-based score estimators (Pattern/Evaluator.h) and their files
# (IO/Binary.cpp)
# ---------------------------------------------------------------------------

# The parameters of the reference's default AccuracyModel (Pattern/Evaluator.h),
# written into estimator files saved without explicit ones.
DEFAULT_ACCURACY = (-0.16594754, 0.95554334, 0.27973529, -0.01616647, 1.28078789)


def estimator_stages(stage_size: int) -> int:
    """Stages(stage_size) (Pattern/Evaluator.cpp:6-9): ceil(65 / stage_size)."""
    return int(L.load().cas_estimator_stages(stage_size))


def _reference_cols(masks) -> int:
    return GroupIndexer(masks, "reference").index_space_size


def save_estimator(path, masks, stage_size: int, weights, accuracy=DEFAULT_ACCURACY) -> None:
    """Save(PatternBasedEstimator) (IO/Binary.cpp:46-63): weights is
    [stages, C] (numpy or tensor, C = the reference-mode columns of masks);
    the file is the reference's, byte for byte."""
    w = weights.detach().cpu().numpy() if isinstance(weights, torch.Tensor) else np.asarray(weights)
    w = np.ascontiguousarray(w, dtype=np.float32)
    stages, cols = estimator_stages(stage_size), _reference_cols(masks)
    if w.shape != (stages, cols):
        raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
    m = np.asarray(masks, dtype=np.uint64)
    a = np.ascontiguousarray(accuracy, dtype=np.float32)
    L.check(L.load().cas_estimator_save(str(path).encode(), stage_size, m.ctypes.data_as(C.c_void_p), len(m),
                                        w.ctypes.data_as(C.c_void_p), a.ctypes.data_as(C.c_void_p), len(a)))


def load_estimator(path) -> dict:
    """LoadPatternBasedEstimator (IO/Binary.cpp:65-68): stage size, the
    stored patterns, the weights [stages, C] and the accuracy parameters."""
    lib = L.load()
    ss, nm, ns, na = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    wps = C.c_int64()
    p = str(path).encode()
    L.check(lib.cas_estimator_file_info(p, C.byref(ss), C.byref(nm), C.byref(ns), C.byref(wps), C.byref(na)))
    masks = np.empty(nm.value, np.uint64)
    w = np.empty((ns.value, wps.value), np.float32)
    acc = np.empty(na.value, np.float32)
    L.check(lib.cas_estimator_file_read(p, masks.ctypes.data_as(C.c_void_p), w.ctypes.data_as(C.c_void_p),
                                        acc.ctypes.data_as(C.c_void_p)))
    return {"stage_size": ss.value, "masks": [int(v) for v in masks], "weights": w, "accuracy": acc.tolist()}


class MultiStageScoreEstimator:
    """MultiStageScoreEstimator (Pattern/Evaluator.cpp:77-88) on the device:
    every stage's dense weights expanded into per-variation tables
    (ScoreEstimator, :11-29), batch evaluation bitwise equal to the
    reference's Eval, and Weights() per stage."""

    def __init__(self, masks, stage_size: int, weights):
        self._lib = L.load()
        self._h = C.c_void_p()
        w = weights if isinstance(weights, torch.Tensor) else torch.from_numpy(np.asarray(weights, np.float32))
        w = w.to(device="cuda", dtype=torch.float32).contiguous()
        stages, cols = estimator_stages(stage_size), _reference_cols(masks)
        if tuple(w.shape) != (stages, cols):
            raise L.SizeMismatch(L.CAS_ERR_SIZE_MISMATCH, "Size mismatch.")
        m = np.asarray(masks, dtype=np.uint64)
        L.check(self._lib.cas_estimator_create(m.ctypes.data_as(C.c_void_p), len(m), stage_size, _ptr(w), _stream(),
                                               C.byref(self._h)))
        ss, st, nm = C.c_int(), C.c_int(), C.c_int()
        wps, tps = C.c_int64(), C.c_int64()
        L.check(self._lib.cas_estimator_info(self._h, C.byref(ss), C.byref(st), C.byref(nm), C.byref(wps),
                                             C.byref(tps)))
        self.stage_size, self.stages, self._n = ss.value, st.value, nm.value
        self.weights_per_stage, self.table_floats = wps.value, tps.value

    @classmethod
    def load(cls, path) -> "MultiStageScoreEstimator":
        f = load_estimator(path)
        return cls(f["masks"], f["stage_size"], f["weights"])

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _sync_before_free()
            self._lib.cas_estimator_destroy(h)
            self._h = None

    def pattern(self) -> list[int]:
        out = np.empty(self._n, np.uint64)
        L.check(self._lib.cas_estimator_patterns(self._h, out.ctypes.data_as(C.c_void_p)))
        return [int(v) for v in out]

    def eval(self, positions: torch.Tensor) -> torch.Tensor:
        _require_cuda(positions, "positions")
        out = torch.empty(positions.shape[0], dtype=torch.float32, device=positions.device)
        L.check(self._lib.cas_estimator_eval(self._h, _ptr(positions), positions.shape[0], _ptr(out), _stream()))
        return out

    def tables(self, stage: int) -> torch.Tensor:
        out = torch.empty(self.table_floats, dtype=torch.float32, device="cuda")
        L.check(self._lib.cas_estimator_tables(self._h, stage, _ptr(out), _stream()))
        return out

    def weights(self, stage: int) -> torch.Tensor:
        out = torch.empty(self.weights_per_stage, dtype=torch.float32, device="cuda")
        L.check(self._lib.cas_estimator_weights(self._h, stage, _ptr(out), _stream()))
        return out

    def save(self, path, accuracy=DEFAULT_ACCURACY) -> None:
        w = torch.stack([self.weights(s) for s in range(self.stages)])
        save_estimator(path, self.pattern(), self.stage_size, w, accuracy)


# ---------------------------------------------------------------------------
# Training-data ingestion
# ---------------------------------------------------------------------------

def _read(fn, path) -> tuple[np.ndarray, np.ndarray]:
    n = C.c_int64()
    p = str(path).encode()
    L.check(fn(p, None, None, 0, C.byref(n)))
    pos = np.empty((n.value, 2), np.uint64)
    sc = np.empty(n.value, np.int8)
    got = C.c_int64()
    L.check(fn(p, pos.ctypes.data_as(C.c_void_p), sc.ctypes.data_as(C.c_void_p), n.value, C.byref(got)))
    return pos[:got.value], sc[:got.value]


def read_records(path) -> tuple[np.ndarray, np.ndarray]:
    """'<QQb' records (NeuralNetwork/NeuralNetwork.py:21-29): positions
    [n, 2] uint64 ({P, O}) and int8 scores."""
    return _read(L.load().cas_read_records, path)


def read_scored_positions(path) -> tuple[np.ndarray, np.ndarray]:
    """Text ScoredPosition lines (IO/File.cpp:16-24): positions [n, 2]
    uint64 and int8 scores."""
    return _read(L.load().cas_read_scored_positions, path)
