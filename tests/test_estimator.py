"""Estimator files (IO/Binary.cpp): the library writes the bytes the
reference's Save writes and reads the reference's files.  Host code only
(no GPU): checked against a file the reference wrote (committed fixture) and,
where the reference tree was compiled here, against the reference itself on
the 5-pattern fitting set."""
import numpy as np
import pytest

import cassandra_b200 as cb
import oracle
from cassandra_b200 import _lib as L

GOLD = np.load("tests/golden/estimator_ref.npz")


def _masks():
    return [int(v) for v in GOLD["masks"]]


def test_stages_follow_reference():
    # Stages(stage_size) = ceil(65 / stage_size), Pattern/Evaluator.cpp:6-9
    for ss in (1, 2, 5, 13, 20, 33, 64, 65, 100):
        assert cb.estimator_stages(ss) == -(-65 // ss)


def test_save_writes_the_reference_bytes(tmp_path):
    p = tmp_path / "est.bin"
    cb.save_estimator(p, _masks(), int(GOLD["stage_size"]), GOLD["weights"], GOLD["accuracy"])
    assert p.read_bytes() == GOLD["file_bytes"].tobytes()


def test_load_reads_the_reference_file(tmp_path):
    p = tmp_path / "ref.bin"
    p.write_bytes(GOLD["file_bytes"].tobytes())
    f = cb.load_estimator(p)
    assert f["stage_size"] == int(GOLD["stage_size"])
    assert f["masks"] == [int(v) for v in GOLD["stored"]]  # the reference stores CreateIndexer's patterns
    np.testing.assert_array_equal(f["weights"], GOLD["weights_back"])
    np.testing.assert_array_equal(np.asarray(f["accuracy"], np.float32), GOLD["accuracy"])


def test_round_trip_through_stored_patterns(tmp_path):
    """Saving what was loaded (stored patterns, same weights) writes the same
    file again."""
    p, q = tmp_path / "a.bin", tmp_path / "b.bin"
    p.write_bytes(GOLD["file_bytes"].tobytes())
    f = cb.load_estimator(p)
    cb.save_estimator(q, f["masks"], f["stage_size"], f["weights"], f["accuracy"])
    assert q.read_bytes() == p.read_bytes()


def test_bad_files_are_rejected(tmp_path):
    blob = GOLD["file_bytes"].tobytes()
    t = tmp_path / "short.bin"
    t.write_bytes(blob[: len(blob) // 2])
    with pytest.raises(cb.CasError):
        cb.load_estimator(t)
    with pytest.raises(cb.CasError):
        cb.load_estimator(tmp_path / "missing.bin")
    with pytest.raises(cb.SizeMismatch):
        cb.save_estimator(tmp_path / "x.bin", _masks(), 33, GOLD["weights"][:1], GOLD["accuracy"])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not compiled here")
def test_five_pattern_file_matches_reference(tmp_path):
    """The 5-pattern fitting set (two of its masks are stored flipped), 5
    stages of seeded weights: byte-identical files both ways."""
    import ctypes as C

    lib = oracle.ref_lib()
    m = np.asarray(cb.PATTERNS_5, np.uint64)
    cols = cb.GroupIndexer(cb.PATTERNS_5, "reference").index_space_size
    ss = 13
    w = np.random.default_rng(5).normal(0, 3, (cb.estimator_stages(ss), cols)).astype(np.float32)
    acc = np.asarray(cb.DEFAULT_ACCURACY, np.float32)
    ref_path, our_path = tmp_path / "ref.bin", tmp_path / "our.bin"
    lib.ref_save_estimator(str(ref_path).encode(), ss, m.ctypes.data_as(C.c_void_p), len(m),
                           w.ctypes.data_as(C.c_void_p), cols, acc.ctypes.data_as(C.c_void_p), len(acc))
    cb.save_estimator(our_path, cb.PATTERNS_5, ss, w)
    assert our_path.read_bytes() == ref_path.read_bytes()
    # the reference loads our file: same stage size, patterns, weights
    ss_o, st_o, na = C.c_int(), C.c_int(), C.c_int()
    masks = np.zeros(8, np.uint64)
    back = np.zeros_like(w)
    got_acc = np.zeros(8, np.float32)
    n = lib.ref_load_estimator(str(our_path).encode(), C.byref(ss_o), C.byref(st_o), masks.ctypes.data_as(C.c_void_p),
                               8, back.ctypes.data_as(C.c_void_p), cols, got_acc.ctypes.data_as(C.c_void_p),
                               C.byref(na))
    assert (ss_o.value, st_o.value, n, na.value) == (ss, len(w), len(m), 5)
    np.testing.assert_array_equal(back, w)
    np.testing.assert_array_equal(got_acc[:5], acc)


def test_entry_points_are_exported():
    lib = L.load()
    for name in ("cas_estimator_stages", "cas_estimator_save", "cas_estimator_file_info", "cas_estimator_file_read",
                 "cas_estimator_create", "cas_estimator_destroy", "cas_estimator_info", "cas_estimator_patterns",
                 "cas_estimator_tables", "cas_estimator_eval", "cas_estimator_weights"):
        assert hasattr(lib, name)
