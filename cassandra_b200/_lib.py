"""ctypes binding of the C ABI declared in include/cassandra_b200.h.

The shared library is built in-tree (``python -m cassandra_b200.build``).  A
missing library is an error: there is no Python or CPU fallback for any of
the compute entry points.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcassandra_b200.so"

# cas_status
CAS_OK = 0
CAS_ERR_SIZE_MISMATCH = 1
CAS_ERR_INVALID_ARGUMENT = 2
CAS_ERR_PATTERN = 3
CAS_ERR_CUDA = 4
CAS_ERR_OUT_OF_MEMORY = 5
CAS_ERR_NO_DEVICE = 6
CAS_ERR_BREAKDOWN = 7
CAS_ERR_NOT_CONVERGED = 8

# enums
CAS_INDEX_REFERENCE = 0
CAS_INDEX_EXPANDED = 1
CAS_F32 = 0
CAS_F64 = 1
CAS_PCG = 0
CAS_LSQR = 1
CAS_LSMR = 3
CAS_CG = 2
CAS_PLAIN_FP64 = 0
CAS_MIXED = 1
CAS_LAYOUT_ROWS = 1
CAS_LAYOUT_BLOCKED = 2


class SolveOpts(C.Structure):
    _fields_ = [
        ("method", C.c_int),
        ("precision", C.c_int),
        ("tol", C.c_double),
        ("max_iterations", C.c_int),
        ("refine_every", C.c_int),
        ("check_every", C.c_int),
        ("jacobi", C.c_int),
        ("scale_columns", C.c_int),
    ]


class SolveReport(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("refinements", C.c_int),
        ("rel_residual", C.c_double),
        ("residuum", C.c_double),
        ("seconds", C.c_double),
        ("setup_seconds", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class AdamOpts(C.Structure):
    """cas_adam_opts: Adam hyperparameters and the objective's L2 weight and Huber threshold."""
    _fields_ = [
        ("lr", C.c_float),
        ("beta1", C.c_float),
        ("beta2", C.c_float),
        ("eps", C.c_float),
        ("l2", C.c_float),
        ("delta", C.c_float),
    ]


class Schedule(C.Structure):
    _fields_ = [
        ("chunks_per_item", C.c_int),
        ("range_major", C.c_int),
        ("items_per_sm", C.c_int),
        ("pack", C.c_int),
        ("persistent", C.c_int),
        ("ms", C.c_float),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class CasError(RuntimeError):
    """A cas_status other than CAS_OK, with the library's message."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{_status_name(status)}: {message}")


class SizeMismatch(CasError, ValueError):
    """CAS_ERR_SIZE_MISMATCH: the reference throws runtime_error("Size mismatch.")."""


_VP = C.c_void_p
_I64 = C.c_int64
_U64 = C.c_uint64
_PP = C.POINTER(C.c_void_p)

# name -> (restype, argtypes)
SIGNATURES: dict[str, tuple] = {
    "cas_status_name": (C.c_char_p, [C.c_int]),
    "cas_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "cas_version": (C.c_int, []),
    "cas_kernel_launches": (C.c_longlong, []),
    "cas_patterns_create": (C.c_int, [_VP, C.c_int, C.c_int, _PP]),
    "cas_patterns_destroy": (None, [_VP]),
    "cas_patterns_cols": (_I64, [_VP]),
    "cas_patterns_nnz_per_row": (C.c_int, [_VP]),
    "cas_patterns_variations": (C.c_int, [_VP, _VP]),
    "cas_patterns_indexer": (C.c_int, [_VP, C.c_int, C.POINTER(_U64), C.POINTER(C.c_int), C.POINTER(_I64),
                                       C.POINTER(_I64)]),
    "cas_index": (C.c_int, [_VP, _VP, _I64, _VP, _VP]),
    "cas_csr_from_positions": (C.c_int, [_VP, _VP, _I64, _VP, _PP]),
    "cas_csr_from_positions_layout": (C.c_int, [_VP, _VP, _I64, C.c_int, _VP, _PP]),
    "cas_csr_layouts": (C.c_int, [_VP]),
    "cas_block_rows": (_I64, []),
    "cas_eval_forward": (C.c_int, [_VP, _I64, _I64, _VP, _VP, _VP]),
    "cas_eval_backward": (C.c_int, [_VP, _I64, _I64, _VP, _VP, _VP]),
    "cas_eval_adam_step": (C.c_int, [_VP, _I64, _I64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "cas_csr_from_indices": (C.c_int, [_VP, C.c_int, _I64, _I64, _VP, _PP]),
    "cas_csr_destroy": (None, [_VP]),
    "cas_csr_rows": (_I64, [_VP]),
    "cas_csr_cols": (_I64, [_VP]),
    "cas_csr_nnz_per_row": (C.c_int, [_VP]),
    "cas_csr_indices": (_VP, [_VP]),
    "cas_csr_transposed": (C.c_int, [_VP, _PP, _PP]),
    "cas_spmv": (C.c_int, [_VP, C.c_int, _VP, _VP, _VP]),
    "cas_spmv_t": (C.c_int, [_VP, C.c_int, _VP, _VP, _VP]),
    "cas_jacobi": (C.c_int, [_VP, C.c_int, _VP, _VP]),
    "cas_solve_opts_default": (None, [C.POINTER(SolveOpts)]),
    "cas_solver_create": (C.c_int, [_VP, C.POINTER(SolveOpts), _VP, _VP, _VP, _PP]),
    "cas_solver_create_normal": (C.c_int, [_VP, C.POINTER(SolveOpts), _VP, _VP, _VP, _PP]),
    "cas_solver_create_normal_diag": (C.c_int, [_VP, C.POINTER(SolveOpts), _VP, _VP, _VP, _VP, _PP]),
    "cas_solver_destroy": (None, [_VP]),
    "cas_solver_iterate": (C.c_int, [_VP, C.c_int]),
    "cas_solver_residuum": (C.c_int, [_VP, C.POINTER(C.c_double)]),
    "cas_solver_x": (C.c_int, [_VP, _VP]),
    "cas_solver_rel_residual": (C.c_int, [_VP, C.POINTER(C.c_double)]),
    "cas_solver_run": (C.c_int, [_VP, C.POINTER(SolveReport)]),
    "cas_solver_iterations": (C.c_int, [_VP]),
    "cas_solver_state_size": (C.c_int, [_VP, C.POINTER(C.c_size_t)]),
    "cas_solver_save_state": (C.c_int, [_VP, _VP, C.c_size_t]),
    "cas_solver_load_state": (C.c_int, [_VP, _VP, C.c_size_t]),
    "cas_solve": (C.c_int, [_VP, C.POINTER(SolveOpts), _VP, _VP, C.POINTER(SolveReport), _VP]),
    "cas_fit_weights": (C.c_int, [_VP, C.c_int, C.c_int, _VP, _VP, _I64, C.POINTER(SolveOpts), _VP,
                                  C.POINTER(SolveReport)]),
    "cas_fit_weights_device": (C.c_int, [_VP, _VP, _VP, _I64, C.POINTER(SolveOpts), _VP, C.POINTER(SolveReport),
                                         _VP]),
    "cas_generate_positions": (C.c_int, [_U64, _I64, C.c_int, C.c_int, _VP, _VP]),
    "cas_generate_positions_host": (C.c_int, [_U64, _I64, _I64, C.c_int, C.c_int, _VP]),
    "cas_generate_targets": (C.c_int, [_VP, _U64, C.c_double, C.c_double, _VP, _VP, _VP]),
    "cas_generate_targets_rows": (C.c_int, [_VP, _U64, C.c_double, C.c_double, _I64, _VP, _VP, _VP]),
    "cas_csr_schedules": (C.c_int, [_VP, _VP, C.c_int, _VP]),
    "cas_cached_memory": (C.c_size_t, []),
    "cas_release_cached_memory": (None, []),
    "cas_csr_from_positions_batched": (C.c_int, [_VP, _VP, _VP, C.c_int, _VP, _VP]),
    "cas_csr_problems": (C.c_int, [_VP, _VP]),
    "cas_solve_batched": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "cas_fit_weights_batched": (C.c_int, [_VP, C.c_int, C.c_int, _VP, _VP, _VP, C.c_int, _VP, _VP, _VP]),
    "cas_fit_weights_batched_device": (C.c_int, [_VP, _VP, _VP, _VP, C.c_int, _VP, _VP, _VP, _VP]),
    "cas_estimator_stages": (C.c_int, [C.c_int]),
    "cas_estimator_save": (C.c_int, [C.c_char_p, C.c_int, _VP, C.c_int, _VP, _VP, C.c_int]),
    "cas_estimator_file_info": (C.c_int, [C.c_char_p, _VP, _VP, _VP, _VP, _VP]),
    "cas_estimator_file_read": (C.c_int, [C.c_char_p, _VP, _VP, _VP]),
    "cas_estimator_create": (C.c_int, [_VP, C.c_int, C.c_int, _VP, _VP, _PP]),
    "cas_estimator_destroy": (None, [_VP]),
    "cas_estimator_info": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "cas_estimator_patterns": (C.c_int, [_VP, _VP]),
    "cas_estimator_tables": (C.c_int, [_VP, C.c_int, _VP, _VP]),
    "cas_estimator_eval": (C.c_int, [_VP, _VP, _I64, _VP, _VP]),
    "cas_estimator_weights": (C.c_int, [_VP, C.c_int, _VP, _VP]),
    "cas_read_records": (C.c_int, [C.c_char_p, _VP, _VP, _I64, _VP]),
    "cas_read_scored_positions": (C.c_int, [C.c_char_p, _VP, _VP, _I64, _VP]),
    "cas_spmv_norm_noalloc_max_rows": (_I64, []),
    "cas_spmv_norm_noalloc": (C.c_int, [_VP, C.c_int, _I64, _I64, _VP, _VP, _VP, _VP]),
}

_lib: C.CDLL | None = None


def load() -> C.CDLL:
    """Loads libcassandra_b200.so (building it first if sources are present
    and the library is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        if os.environ.get("CASSANDRA_B200_NO_BUILD"):
            raise ImportError(f"{LIB_PATH} is missing; run `python -m cassandra_b200.build`")
        from . import build as _build

        _build.build()
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _status_name(status: int) -> str:
    try:
        return load().cas_status_name(status).decode()
    except Exception:  # pragma: no cover - only when the library itself is broken
        return f"status {status}"


def last_error() -> str:
    lib = load()
    buf = C.create_string_buffer(4096)
    lib.cas_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    """Raises CasError (SizeMismatch for size errors) unless status is CAS_OK."""
    if status == CAS_OK:
        return
    msg = last_error()
    if status == CAS_ERR_SIZE_MISMATCH:
        raise SizeMismatch(status, msg)
    raise CasError(status, msg)
