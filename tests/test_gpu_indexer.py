"""Indexer kernel parity: bit-exact with the reference GroupIndexer (golden
vectors from the reference, the compiled reference where present, and the C
oracle for the expanded mode)."""
import numpy as np
import pytest
import torch

import cassandra_b200 as cb
from tests.golden.make_golden import FIXTURES, SET5, SET8

pytestmark = pytest.mark.gpu


def _dev(pos: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(pos).view(np.int64).reshape(-1, 2)).cuda()


def _u32(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("name", list(FIXTURES) + ["mix", "set5", "set8"])
def test_indices_match_reference_golden(cuda, golden_indexer, name):
    masks = golden_indexer[f"masks_{name}"]
    g = cb.GroupIndexer(masks, "reference")
    assert g.index_space_size == int(golden_indexer[f"cols_{name}"])
    np.testing.assert_array_equal(g.variations(), golden_indexer[f"variations_{name}"])
    got = _u32(g.indices(_dev(golden_indexer["positions"])))
    np.testing.assert_array_equal(got, golden_indexer[f"idx_{name}"])


@pytest.mark.parametrize("mode", ["reference", "expanded"])
@pytest.mark.parametrize("n", [1, 31, 33, 1000, 100_003])
def test_indices_match_oracle_random_play(cuda, orc, mode, n):
    pos = cb.generate_positions(99 + n, n, 4, 56)
    host = pos.cpu().numpy().view(np.uint64)
    for masks in (SET5, SET8, list(FIXTURES.values())):
        g = cb.GroupIndexer(masks, mode)
        want = orc.group_index(masks, 0 if mode == "reference" else 1, host)
        np.testing.assert_array_equal(_u32(g.indices(pos)), want)


def test_indices_match_compiled_reference(cuda, ref):
    import ctypes as C

    pos = cb.generate_positions(5, 50_000, 0, 60)
    host = np.ascontiguousarray(pos.cpu().numpy().view(np.uint64))
    for masks in (SET8, list(FIXTURES.values())):
        m = np.asarray(masks, np.uint64)
        cols = np.zeros(1, np.int64)
        lib = ref.ref_lib()
        k = lib.ref_group_info(m.ctypes.data_as(C.c_void_p), len(m), cols.ctypes.data_as(C.c_void_p), None)
        want = np.empty((len(host), k), np.uint32)
        lib.ref_group_index(m.ctypes.data_as(C.c_void_p), len(m), host.ctypes.data_as(C.c_void_p), len(host),
                            want.ctypes.data_as(C.c_void_p))
        got = _u32(cb.GroupIndexer(masks, "reference").indices(pos))
        np.testing.assert_array_equal(got, want)


def test_indices_of_empty_batch(cuda):
    g = cb.GroupIndexer(SET5)
    out = g.indices(torch.empty((0, 2), dtype=torch.int64, device="cuda"))
    assert out.shape == (0, g.nnz_per_row)


def test_indices_cover_index_space_of_all_configurations(cuda, ref):
    """PatternTest/Indexer.cpp:51-92 on the device."""
    import ctypes as C

    for name, m in FIXTURES.items():
        n = ref.ref_lib().ref_configurations(m, None)
        conf = np.empty((n, 2), np.uint64)
        ref.ref_lib().ref_configurations(m, conf.ctypes.data_as(C.c_void_p))
        g = cb.GroupIndexer([m])
        got = np.unique(_u32(g.indices(_dev(conf))))
        np.testing.assert_array_equal(got, np.arange(g.index_space_size, dtype=np.uint32))


def test_symmetry_invariance_on_device(cuda, orc, golden_indexer):
    """PatternTest/Indexer.cpp:8-47: sorted index multisets equal under the 8 symmetries."""
    pos = golden_indexer["positions"][:2000]
    lib = orc.c_lib()

    def flip(w, a):
        return np.array([[lib.or_flip(w, int(p)), lib.or_flip(w, int(o))] for p, o in a], dtype=np.uint64)

    variants = [flip(0, pos), flip(1, pos), flip(2, pos), flip(3, pos), flip(0, flip(2, pos)),
                flip(1, flip(2, pos)), flip(3, flip(2, pos))]
    for mode in ("reference", "expanded"):
        g = cb.GroupIndexer(list(FIXTURES.values()), mode)
        base = np.sort(_u32(g.indices(_dev(pos))), axis=1)
        for v in variants:
            np.testing.assert_array_equal(np.sort(_u32(g.indices(_dev(v))), axis=1), base)


def test_generator_device_equals_host(cuda):
    d = cb.generate_positions(1234, 5000, 20, 40).cpu().numpy().view(np.uint64)
    h = cb.generate_positions_host(1234, 0, 5000, 20, 40)
    np.testing.assert_array_equal(d, h)
    empties = 64 - np.array([bin(int(p) | int(o)).count("1") for p, o in h])
    assert empties.min() >= 20 and empties.max() <= 40
    assert np.all((h[:, 0] & h[:, 1]) == 0)


@pytest.mark.parametrize("layout", ["rows", "blocked"])
def test_device_inputs_equal_oracle_restatement(cuda, orc, layout):
    """The benchmark's reference arm builds its inputs with the oracle's C
    restatement of the generator (no CUDA library in that process): the
    positions and the targets b equal the device generator's bit for bit."""
    pos = cb.generate_positions(2024, 200_000, 20, 40)
    np.testing.assert_array_equal(pos.cpu().numpy().view(np.uint64), orc.generate_positions(2024, 0, 200_000, 20, 40))
    g = cb.GroupIndexer(SET8, "expanded")
    a = cb.MatrixCSR.from_positions(g, pos, layout)
    b = cb.generate_targets(a, 2024).cpu().numpy()
    idx = orc.group_index(SET8, 1, pos.cpu().numpy().view(np.uint64))
    want, _ = orc.generate_targets(idx, g.index_space_size, 2024)
    np.testing.assert_array_equal(b, want)
