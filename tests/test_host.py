"""Host-side checks that need no GPU: the C ABI library loads and exports
every declared symbol, pattern-set metadata equals the reference's, argument
validation, and the CPU-only legs of the benchmark."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import cassandra_b200 as cb
from cassandra_b200 import _lib as L
from tests.golden.make_golden import FIXTURES, SET5, SET8

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"CAS_API\s+[^;(]*?\b(cas_\w+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"cas_index", "cas_spmv", "cas_spmv_t", "cas_jacobi", "cas_solver_create", "cas_fit_weights"} <= names


def test_library_exports_every_declared_symbol():
    lib = L.load()
    for name in sorted(declared_symbols()):
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_bindings_cover_every_declared_symbol():
    assert declared_symbols() <= set(L.SIGNATURES), declared_symbols() - set(L.SIGNATURES)


@pytest.mark.parametrize("name", list(FIXTURES) + ["mix", "set5", "set8"])
def test_pattern_metadata_matches_reference(golden_indexer, name):
    masks = golden_indexer[f"masks_{name}"]
    g = cb.GroupIndexer(masks, "reference")
    assert g.index_space_size == int(golden_indexer[f"cols_{name}"])
    assert g.nnz_per_row == golden_indexer[f"idx_{name}"].shape[1]
    np.testing.assert_array_equal(g.variations(), golden_indexer[f"variations_{name}"])


def test_create_indexer_facts_match_reference(golden_indexer):
    for m, stored, order, space in golden_indexer["create_indexer"]:
        g = cb.GroupIndexer([int(m)], "reference")
        info = g.indexer(0)
        assert (info["pattern"], info["order"], info["space"]) == (int(stored), int(order), int(space))


def test_expanded_sizes():
    g = cb.GroupIndexer(SET5, "expanded")
    assert (g.index_space_size, g.nnz_per_row) == (150_903, 40)
    g = cb.GroupIndexer(SET8, "expanded")
    assert (g.index_space_size, g.nnz_per_row) == (166_212, 64)
    offs = [g.indexer(i)["offset"] for i in range(8)]
    assert offs == list(np.cumsum([0] + [3 ** bin(m).count("1") for m in SET8[:-1]]))


@pytest.mark.parametrize("bad", [[0], [0xFFFFFFFF0], [(1 << 17) - 1]])
def test_unusable_masks_are_rejected(bad):
    with pytest.raises(cb.CasError) as e:
        cb.GroupIndexer(bad)
    assert e.value.status == L.CAS_ERR_PATTERN


def test_invalid_arguments_are_reported():
    lib = L.load()
    h = C.c_void_p()
    assert lib.cas_patterns_create(None, 0, 0, C.byref(h)) == L.CAS_ERR_INVALID_ARGUMENT
    assert "cas_patterns_create" in L.last_error()
    m = np.array([0x42FF], np.uint64)
    assert lib.cas_patterns_create(m.ctypes.data_as(C.c_void_p), 1, 7, C.byref(h)) == L.CAS_ERR_INVALID_ARGUMENT
    assert lib.cas_status_name(L.CAS_ERR_SIZE_MISMATCH) == b"CAS_ERR_SIZE_MISMATCH"
    o = cb.solve_opts()
    o.method = 9
    assert lib.cas_solver_create(None, C.byref(o), None, None, None, C.byref(h)) == L.CAS_ERR_INVALID_ARGUMENT
    # batches: 1 to 64 problems of non-negative size, checked before any device work
    g = cb.GroupIndexer(SET8, "expanded")
    for sizes in ([], [1] * 65, [3, -1]):
        rows = np.asarray(sizes or [0], np.int64)
        st = lib.cas_csr_from_positions_batched(g.handle, None, rows.ctypes.data_as(C.c_void_p), len(sizes), None,
                                                C.byref(h))
        assert st == L.CAS_ERR_INVALID_ARGUMENT, sizes
    assert lib.cas_solve_batched(None, C.byref(cb.solve_opts()), None, None, None, None) == L.CAS_ERR_INVALID_ARGUMENT
    # the evaluator's training step needs a blocked CSR
    opts = L.AdamOpts(1e-2, 0.9, 0.999, 1e-8, 1e-4, 4.0)
    st = lib.cas_eval_adam_step(None, 0, 0, None, None, None, None, None, None, C.byref(opts), None)
    assert st == L.CAS_ERR_INVALID_ARGUMENT and "cas_eval_adam_step" in L.last_error()


def test_no_cpu_fallback_without_a_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = L.load()
    g = cb.GroupIndexer(SET5)
    pos = np.zeros((4, 2), np.uint64)
    out = np.zeros((4, g.nnz_per_row), np.uint32)
    st = lib.cas_index(g.handle, pos.ctypes.data_as(C.c_void_p), 4, out.ctypes.data_as(C.c_void_p), None)
    assert st == L.CAS_ERR_NO_DEVICE
    assert "no CPU fallback" in L.last_error()
    w = np.zeros(g.index_space_size, np.float32)
    with pytest.raises(cb.CasError) as e:
        cb.fit_weights(SET5, pos, np.zeros(4, np.float32))
    assert e.value.status == L.CAS_ERR_NO_DEVICE
    del w


def test_host_generator_is_deterministic_and_legal(ref):
    a = cb.generate_positions_host(42, 0, 2000, 1, 60)
    b = cb.generate_positions_host(42, 1000, 1000, 1, 60)
    np.testing.assert_array_equal(a[1000:], b)
    assert np.all((a[:, 0] & a[:, 1]) == 0)
    lib = ref.ref_lib()
    # every position is reachable: its side to move or the opponent can move,
    # unless the board is full; and discs + empties add up
    for p, o in a[:300]:
        empt = 64 - bin(int(p) | int(o)).count("1")
        assert 1 <= empt <= 60
        if empt > 0:
            assert lib.ref_possible_moves(int(p), int(o)) or lib.ref_possible_moves(int(o), int(p)) or empt == 0


def test_reference_expanded_index_matches_oracle(ref, orc):
    lib = ref.ref_lib()
    lib.ref_expanded_index.restype = None
    lib.ref_expanded_index.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p]
    pos = cb.generate_positions_host(3, 0, 4000, 10, 50)
    m = np.array(SET8, np.uint64)
    out = np.empty((len(pos), 64), np.uint32)
    lib.ref_expanded_index(m.ctypes.data_as(C.c_void_p), 8, pos.ctypes.data_as(C.c_void_p), len(pos),
                           out.ctypes.data_as(C.c_void_p))
    np.testing.assert_array_equal(out, orc.group_index(m, 1, pos))


def test_reference_arm_runs_on_cpu(ref):
    import bench

    args = bench.parse_args(["--impl", "reference", "--steps", "1", "--warmup", "0", "--cpu-sample-rows", "3000",
                             "--rows", "30000"])
    res = bench.run_reference(args)
    assert res["impl"] == "reference" and res["value"] > 0
    assert res["e2e"]["h2d_bytes_per_step"] == 0
    assert res["cpu_baseline"]["kind"] == "reference"
    # the same workload description as the GPU arm, the whole workload every step
    assert res["config"] == bench.single_config(args)
    assert res["breakdown"]["rel_residual"] <= 1e-8
    assert "30000 rows" in res["cpu_baseline"]["sample"]


def test_reference_arm_loads_no_cuda_library(ref):
    """The reference arm's process builds its inputs with the oracle's
    restatement of the generator and maps only the oracle's libraries."""
    import subprocess
    import sys

    code = ("import bench; a = bench.parse_args(['--impl', 'reference', '--steps', '1', '--warmup', '0', "
            "'--rows', '5000']); r = bench.run_reference(a); assert r['value'] > 0; "
            "print('\\n'.join(sorted({l.split()[-1] for l in open('/proc/self/maps') if '.so' in l})))")
    out = subprocess.run([sys.executable, "-c", code], cwd=str(ROOT), capture_output=True, text=True, check=True)
    mine = [l for l in out.stdout.splitlines() if l.startswith(str(ROOT))]
    assert mine and all("/oracle/_ref/" in l or "/oracle/_build/" in l for l in mine), mine


def test_reference_check_pins_a_solution(ref, orc):
    """The bench's oracle check: the oracle's own PCG solution of the system
    passes with a residual below the tolerance and weights within rounding
    of the reference's FP64 PCG on the columns with entries."""
    import bench

    args = bench.parse_args(["--rows", "20000"])
    pos = orc.generate_positions(args.seed, 0, args.rows, args.min_empties, args.max_empties)
    idx = orc.group_index(bench.PATTERNS_8, 1, pos)
    b, _ = orc.generate_targets(idx, bench.COLS_8, args.seed)
    x, _, _ = orc.pcg(idx, bench.COLS_8, b, 20000, tol=1e-10, check_every=10)
    cpu, check = bench.reference_check(args, pos, b, {"oracle_pcg": x})
    assert cpu["kind"] == "reference" and cpu["value"] > 0
    assert check["oracle_pcg"]["rel_residual_fp64"] <= 1e-9
    assert check["reference"]["rel_residual_fp64"] <= 1e-8
    assert check["oracle_pcg"]["max_weight_err_hit_rel"] < 1e-3
    assert 0 < check["hit_cols"] < bench.COLS_8


def test_reference_arm_runs_the_evaluator_workload_on_cpu(ref):
    """The evaluator workload's reference arm: the reference's products on
    kept per-minibatch matrices plus numpy loss and Adam, scaled to the
    epoch."""
    import bench

    args = bench.parse_args(["--impl", "reference", "--workload", "evaluator", "--steps", "1", "--warmup", "0",
                             "--eval-rows", "200000", "--eval-sample-batches", "1"])
    res = bench.run_reference(args)
    assert res["impl"] == "reference" and res["value"] > 0 and res["metric"] == bench.EVAL_METRIC
    assert res["config"]["rows"] == 200000
    assert "1 of 4 minibatches" in res["cpu_baseline"]["sample"]


def test_graph_buffer_guard_logic():
    """The evaluator's guard for buffers that captured CUDA graphs use: once
    a Trainer captured over n blocks per call, a call over more is refused."""
    from cassandra_b200 import evaluator as ev

    class Csr:
        pass

    c = Csr()
    ev._guard_graph_buffers(c, 100)  # no graphs captured: anything goes
    c._graph_blocks = 4
    ev._guard_graph_buffers(c, 4)
    with pytest.raises(RuntimeError, match="reallocate"):
        ev._guard_graph_buffers(c, 5)
    assert ev._blocks_spanned(0, 65536, 16384) == 4
    assert ev._blocks_spanned(6 * 16384, 6 * 16384 + 1000, 16384) == 1
    assert ev._blocks_spanned(7, 7, 16384) == 0
