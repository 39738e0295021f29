"""Parity oracle — TEST INFRASTRUCTURE ONLY.

Two checkers live here, both CPU-only and both used only by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg:

* ``c``   — the C restatement in oracle.c (FP64), built by ``make -C oracle
  oracle`` into oracle/_build/liboracle.so.  Always available.
* ``ref`` / ``ref64`` — the reference's own sources compiled where they lie
  (FP32 as shipped, and the Math/ sources retyped to FP64), built by ``make -C
  oracle ref`` into oracle/_ref/ when the reference tree is present.  Those
  libraries travel with the repository snapshot; the reference tree does not.

The shipped library never imports this package.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libcasref.so"
REF64_SO = HERE / "_ref" / "libcasref64.so"
# the reference tree: $CASSANDRA_REFERENCE when set, else its location in the build container
REFERENCE_TREE = Path(os.environ.get("CASSANDRA_REFERENCE", "/root/reference"))

_VP = C.c_void_p
_I64 = C.c_int64


def build(ref: bool = True) -> None:
    """Builds liboracle.so, and the reference libraries when the tree exists."""
    targets = ["oracle"]
    if ref and REFERENCE_TREE.is_dir():
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", str(HERE), f"REF={REFERENCE_TREE}", *targets], check=True)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_VP)


_c = None
_ref = None
_ref64 = None


def c_lib() -> C.CDLL:
    global _c
    if _c is None:
        if not ORACLE_SO.exists():
            build(ref=False)
        lib = C.CDLL(str(ORACLE_SO))
        lib.or_flip.restype = C.c_uint64
        lib.or_flip.argtypes = [C.c_int, C.c_uint64]
        lib.or_fast_index.restype = C.c_uint32
        lib.or_fast_index.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        lib.or_group_info.restype = C.c_int
        lib.or_group_info.argtypes = [_VP, C.c_int, C.c_int, C.POINTER(_I64), C.POINTER(C.c_int)]
        lib.or_group_index.restype = C.c_int
        lib.or_group_index.argtypes = [_VP, C.c_int, C.c_int, _VP, _I64, _VP]
        for n in ("or_spmv", "or_spmv_t", "or_jacobi"):
            getattr(lib, n).restype = None
        lib.or_spmv.argtypes = [C.c_int, _I64, _I64, _VP, _VP, _VP]
        lib.or_spmv_t.argtypes = [C.c_int, _I64, _I64, _VP, _VP, _VP]
        lib.or_jacobi.argtypes = [C.c_int, _I64, _I64, _VP, _VP]
        lib.or_normal_residual.restype = C.c_double
        lib.or_normal_residual.argtypes = [C.c_int, _I64, _I64, _VP, _VP, _VP]
        lib.or_pcg.restype = C.c_int
        lib.or_pcg.argtypes = [C.c_int, _I64, _I64, _VP, _VP, C.c_int, C.c_int, C.c_double, C.c_int, _VP,
                               C.POINTER(C.c_double)]
        for n in ("or_lsqr", "or_lsmr"):
            getattr(lib, n).restype = C.c_int
            getattr(lib, n).argtypes = [C.c_int, _I64, _I64, _VP, _VP, C.c_int, C.c_double, C.c_int, _VP,
                                        C.POINTER(C.c_double)]
        for n in ("or_lsqr_scaled", "or_lsmr_scaled"):
            getattr(lib, n).restype = C.c_int
            getattr(lib, n).argtypes = [C.c_int, _I64, _I64, _VP, _VP, C.c_int, C.c_int, C.c_double, C.c_int, _VP,
                                        C.POINTER(C.c_double)]
        lib.or_generate_positions.restype = C.c_int
        lib.or_generate_positions.argtypes = [C.c_uint64, _I64, _I64, C.c_int, C.c_int, _VP]
        lib.or_generate_targets.restype = None
        lib.or_generate_targets.argtypes = [C.c_int, _I64, _I64, _VP, C.c_uint64, C.c_double, C.c_double, _VP, _VP]
        _c = lib
    return _c


def ref_available() -> bool:
    return REF_SO.exists() and REF64_SO.exists()


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference tree)")
        lib = C.CDLL(str(REF_SO))
        lib.ref_flip.restype = C.c_uint64
        lib.ref_flip.argtypes = [C.c_int, C.c_uint64]
        lib.ref_fast_index.restype = C.c_uint32
        lib.ref_fast_index.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        lib.ref_create_indexer.restype = None
        lib.ref_create_indexer.argtypes = [C.c_uint64, _VP, _VP, _VP]
        lib.ref_group_info.restype = C.c_int
        lib.ref_group_info.argtypes = [_VP, C.c_int, _VP, _VP]
        lib.ref_group_index.restype = None
        lib.ref_group_index.argtypes = [_VP, C.c_int, _VP, _I64, _VP]
        lib.ref_indexer_indices.restype = C.c_int
        lib.ref_indexer_indices.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, _VP]
        lib.ref_random_positions.restype = None
        lib.ref_random_positions.argtypes = [C.c_uint, _I64, _VP]
        lib.ref_configurations.restype = _I64
        lib.ref_configurations.argtypes = [C.c_uint64, _VP]
        lib.ref_possible_moves.restype = C.c_uint64
        lib.ref_possible_moves.argtypes = [C.c_uint64, C.c_uint64]
        lib.ref_play.restype = None
        lib.ref_play.argtypes = [C.c_uint64, C.c_uint64, C.c_int, _VP]
        for n in ("ref_spmv", "ref_spmv_t"):
            getattr(lib, n).restype = None
            getattr(lib, n).argtypes = [C.c_int, _I64, _I64, _VP, _VP, _VP]
        lib.ref_csr_new.restype = _VP
        lib.ref_csr_new.argtypes = [C.c_int, _I64, _I64, _VP]
        lib.ref_csr_free.restype = None
        lib.ref_csr_free.argtypes = [_VP]
        for n in ("ref_csr_mul", "ref_csr_tmul"):
            getattr(lib, n).restype = None
            getattr(lib, n).argtypes = [_VP, _VP, _VP]
        lib.ref_jacobi.restype = None
        lib.ref_jacobi.argtypes = [C.c_int, _I64, _I64, _VP, _VP]
        for n in ("ref_pcg", "ref_lsqr", "ref_lsmr"):
            getattr(lib, n).restype = None
            getattr(lib, n).argtypes = [C.c_int, _I64, _I64, _VP, _VP, C.c_int, _VP, _VP]
        lib.ref_estimator_eval.restype = None
        lib.ref_estimator_eval.argtypes = [_VP, C.c_int, _VP, _I64, _VP, _I64, _VP]
        lib.ref_estimator_weights.restype = None
        lib.ref_estimator_weights.argtypes = [_VP, C.c_int, _VP, _I64, _VP]
        lib.ref_msse_eval.restype = None
        lib.ref_msse_eval.argtypes = [C.c_int, _VP, C.c_int, _VP, _I64, _VP, _I64, _VP]
        lib.ref_save_estimator.restype = None
        lib.ref_save_estimator.argtypes = [C.c_char_p, C.c_int, _VP, C.c_int, _VP, _I64, _VP, C.c_int]
        lib.ref_parse_scored_position.restype = C.c_int
        lib.ref_parse_scored_position.argtypes = [C.c_char_p, _VP, _VP, _VP]
        lib.ref_format_scored_position.restype = None
        lib.ref_format_scored_position.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_char_p]
        lib.ref_load_estimator.restype = C.c_int
        lib.ref_load_estimator.argtypes = [C.c_char_p, _VP, _VP, _VP, C.c_int, _VP, _I64, _VP, _VP]
        _ref = lib
    return _ref


@contextlib.contextmanager
def single_thread():
    """Runs the compiled reference on one OpenMP thread: its `x * A`
    (Math/MatrixCSR.cpp:67-87) merges thread sums in arrival order, so only a
    single thread gives a reproducible target."""
    gomp = C.CDLL("libgomp.so.1")
    before = gomp.omp_get_max_threads()
    gomp.omp_set_num_threads(1)
    try:
        yield
    finally:
        gomp.omp_set_num_threads(before)


def ref64_lib() -> C.CDLL:
    global _ref64
    if _ref64 is None:
        if not REF64_SO.exists():
            raise FileNotFoundError(f"{REF64_SO} not built (needs the reference tree)")
        lib = C.CDLL(str(REF64_SO))
        for n in ("ref64_spmv", "ref64_spmv_t"):
            getattr(lib, n).restype = None
            getattr(lib, n).argtypes = [C.c_int, _I64, _I64, _VP, _VP, _VP]
        lib.ref64_jacobi.restype = None
        lib.ref64_jacobi.argtypes = [C.c_int, _I64, _I64, _VP, _VP]
        for n in ("ref64_pcg", "ref64_lsqr", "ref64_lsmr"):
            getattr(lib, n).restype = C.c_int
            getattr(lib, n).argtypes = [C.c_int, _I64, _I64, _VP, _VP, C.c_int, C.c_double, C.c_int, _VP, _VP, _VP]
        lib.ref64_check.restype = None
        lib.ref64_check.argtypes = [C.c_int, _I64, _I64, _VP, _VP, C.c_int, _VP, _VP, _VP]
        lib.ref64_pcg_seconds_per_iteration.restype = C.c_double
        lib.ref64_pcg_seconds_per_iteration.argtypes = [C.c_int, _I64, _I64, _VP, _VP, C.c_int]
        _ref64 = lib
    return _ref64


# ---------------------------------------------------------------- C oracle --

def group_info(masks, mode: int) -> tuple[int, int]:
    m = np.ascontiguousarray(masks, dtype=np.uint64)
    cols, k = _I64(), C.c_int()
    if c_lib().or_group_info(_p(m), len(m), mode, C.byref(cols), C.byref(k)) != 0:
        raise ValueError("unusable mask")
    return cols.value, k.value


def group_index(masks, mode: int, positions: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(masks, dtype=np.uint64)
    pos = np.ascontiguousarray(positions, dtype=np.uint64).reshape(-1, 2)
    _, k = group_info(m, mode)
    out = np.empty((len(pos), k), dtype=np.uint32)
    if c_lib().or_group_index(_p(m), len(m), mode, _p(pos), len(pos), _p(out)) != 0:
        raise ValueError("unusable mask")
    return out


def spmv(idx: np.ndarray, cols: int, x: np.ndarray) -> np.ndarray:
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty(idx.shape[0], dtype=np.float64)
    c_lib().or_spmv(idx.shape[1], idx.shape[0], cols, _p(idx), _p(x), _p(y))
    return y


def spmv_t(idx: np.ndarray, cols: int, y: np.ndarray) -> np.ndarray:
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    y = np.ascontiguousarray(y, dtype=np.float64)
    x = np.empty(cols, dtype=np.float64)
    c_lib().or_spmv_t(idx.shape[1], idx.shape[0], cols, _p(idx), _p(y), _p(x))
    return x


def jacobi(idx: np.ndarray, cols: int) -> np.ndarray:
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    d = np.empty(cols, dtype=np.float64)
    with np.errstate(divide="ignore"):
        c_lib().or_jacobi(idx.shape[1], idx.shape[0], cols, _p(idx), _p(d))
    return d


def normal_residual(idx: np.ndarray, cols: int, b: np.ndarray, x: np.ndarray) -> float:
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    return c_lib().or_normal_residual(idx.shape[1], idx.shape[0], cols, _p(idx), _p(b), _p(x))


def pcg(idx, cols, b, iterations, tol=0.0, check_every=1, jacobi=True):
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.empty(cols, dtype=np.float64)
    res = C.c_double()
    it = c_lib().or_pcg(idx.shape[1], idx.shape[0], cols, _p(idx), _p(b), int(jacobi), iterations, tol,
                        check_every, _p(x), C.byref(res))
    return x, res.value, it


def lsqr(idx, cols, b, iterations, tol=0.0, check_every=1, scale=False):
    """LSQR (Math/Solver.h:128-182) in FP64 from x0 = 0: x, phi_bar, steps.
    scale=True: on A S, S = diag(A'A)^-1/2, x = S y (not in the reference)."""
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.empty(cols, dtype=np.float64)
    res = C.c_double()
    it = c_lib().or_lsqr_scaled(idx.shape[1], idx.shape[0], cols, _p(idx), _p(b), int(scale), iterations, tol,
                                check_every, _p(x), C.byref(res))
    return x, res.value, it


def lsmr(idx, cols, b, iterations, tol=0.0, check_every=1, scale=False):
    """LSMR (Math/Solver.h:222-287) in FP64 from x0 = 0: x, |zeta_bar|, steps.
    scale=True: on A S, S = diag(A'A)^-1/2, x = S y (not in the reference)."""
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.empty(cols, dtype=np.float64)
    res = C.c_double()
    it = c_lib().or_lsmr_scaled(idx.shape[1], idx.shape[0], cols, _p(idx), _p(b), int(scale), iterations, tol,
                                check_every, _p(x), C.byref(res))
    return x, res.value, it


def generate_positions(seed: int, first: int, n: int, min_empties: int, max_empties: int) -> np.ndarray:
    """The library's seeded random-play positions, restated in C: uint64 [n, 2]
    rows (P, O) for position indices first .. first + n - 1."""
    out = np.empty((n, 2), dtype=np.uint64)
    if c_lib().or_generate_positions(seed, first, n, min_empties, max_empties, _p(out)) != 0:
        raise ValueError("bad arguments or an unreachable empty count")
    return out


def generate_targets(idx: np.ndarray, cols: int, seed: int, w_sigma: float = 0.5,
                     noise_sigma: float = 4.0) -> tuple[np.ndarray, np.ndarray]:
    """The library's seeded targets for the system idx, restated in C:
    (b, w_true) with b = clamp(2 rint((A w* + e) / 2), -64, 64)."""
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    b = np.empty(idx.shape[0], dtype=np.float64)
    w = np.empty(cols, dtype=np.float64)
    c_lib().or_generate_targets(idx.shape[1], idx.shape[0], cols, _p(idx), seed, w_sigma, noise_sigma, _p(b), _p(w))
    return b, w
