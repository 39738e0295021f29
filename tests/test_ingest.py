"""Training-data ingestion (host code): '<QQb' records as the reference's
Python reader unpacks them (NeuralNetwork/NeuralNetwork.py:21-29) and text
ScoredPosition lines as the reference's ScoredPosition::FromString parses
them (Game/ScoredPosition.cpp:3-8), checked against struct.unpack and, where
the reference tree was compiled here, against the reference's parser."""
import ctypes as C
import struct

import numpy as np
import pytest

import cassandra_b200 as cb
import oracle


def _positions(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 2**64, n, dtype=np.uint64)
    b = rng.integers(0, 2**64, n, dtype=np.uint64)
    return np.stack([a & ~b, ~a & b], axis=1)


def test_records_match_struct_unpack(tmp_path):
    pos = _positions(1000, 1)
    sc = np.random.default_rng(2).integers(-64, 65, 1000).astype(np.int8)
    blob = b"".join(struct.pack("<QQb", int(p), int(o), int(s)) for (p, o), s in zip(pos, sc))
    f = tmp_path / "e20.psc"
    f.write_bytes(blob + b"\x01\x02\x03")  # a trailing partial record is not read
    got_pos, got_sc = cb.read_records(f)
    want = [struct.unpack("<QQb", blob[i:i + 17]) for i in range(0, len(blob), 17)]
    np.testing.assert_array_equal(got_pos, np.array([[p, o] for p, o, _ in want], np.uint64))
    np.testing.assert_array_equal(got_sc, np.array([s for _, _, s in want], np.int8))


def test_empty_and_missing_record_files(tmp_path):
    f = tmp_path / "empty.psc"
    f.write_bytes(b"")
    p, s = cb.read_records(f)
    assert p.shape == (0, 2) and s.shape == (0,)
    with pytest.raises(cb.CasError):
        cb.read_records(tmp_path / "missing.psc")


def _line(p, o, side_x, score_text):
    board = []
    x, y = (p, o) if side_x else (o, p)
    for i in range(64):
        bit = 1 << (63 - i)
        board.append("X" if x & bit else ("O" if y & bit else "-"))
    return "".join(board) + " " + ("X" if side_x else "O") + " % " + score_text


def _lines(n, seed):
    rng = np.random.default_rng(seed)
    pos = _positions(n, seed)
    out = []
    for i, (p, o) in enumerate(pos):
        s = int(rng.integers(-64, 65))
        text = ("+" if s >= 0 else "-") + f"{abs(s):02d}"
        if i % 7 == 3:
            text = f"{s:+d}"  # other digit counts
        out.append((int(p), int(o), bool(rng.integers(0, 2)), text))
    return out


def test_scored_position_lines(tmp_path):
    rows = _lines(500, 3)
    f = tmp_path / "pos.txt"
    f.write_text("\n".join(_line(*r) for r in rows) + "\n")
    pos, sc = cb.read_scored_positions(f)
    assert len(pos) == len(rows)
    for (p, o, side_x, text), got_p, got_s in zip(rows, pos, sc):
        assert int(got_p[0]) == p and int(got_p[1]) == o  # the side to move becomes P
        v = int(text[1:])
        want = -(v // 2) if text[0] == "-" else v // 2
        assert int(got_s) == want


def test_bad_lines_are_errors(tmp_path):
    f = tmp_path / "bad.txt"
    good = _line(1, 2, True, "+10")
    f.write_text(good + "\n" + good[:60] + "\n")
    with pytest.raises(cb.CasError, match="line 2"):
        cb.read_scored_positions(f)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not compiled here")
def test_lines_match_reference_parser(tmp_path):
    lib = oracle.ref_lib()
    rows = _lines(2000, 9)
    text = [_line(*r) for r in rows]
    # the reference's own formatting of scored positions parses the same way
    buf = C.create_string_buffer(96)
    for p, o in _positions(50, 10):
        lib.ref_format_scored_position(int(p), int(o), int(np.int8(int(p) % 65 - 32)), buf)
        text.append(buf.value.decode())
    f = tmp_path / "pos.txt"
    f.write_text("\r\n".join(text))  # CRLF and no final newline
    pos, sc = cb.read_scored_positions(f)
    assert len(pos) == len(text)
    for line, gp, gs in zip(text, pos, sc):
        p, o, s = C.c_uint64(), C.c_uint64(), C.c_int()
        assert lib.ref_parse_scored_position(line.encode(), C.byref(p), C.byref(o), C.byref(s)) == 0
        assert (int(gp[0]), int(gp[1]), int(gs)) == (p.value, o.value, s.value)
