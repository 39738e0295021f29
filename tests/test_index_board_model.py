"""A CPU model of the indexers' digit boards (cassandra_b200/csrc/indexer.cuh:
fill_board, board_digits; cassandra_b200/csrc/core.cu: cell_word).

A position's cell at square t is (P >> t & 1) + 2 (O >> t & 1).  The ROWS
indexer has lanes 0-15 of a warp write the 64 cells as 16 words, lane j's
word holding squares 4j .. 4j+3 in its bytes, spread from the two nibbles by
one multiply each; the BLOCKED indexer writes one byte per square into
lines of STRIDE bytes.  Both are checked against the per-square cells, and
the digits read back from them against the oracle's indices.  CPU only."""
import numpy as np


def cell_word(p_nib: int, o_nib: int) -> int:
    sp = (p_nib * 0x00204081) & 0x01010101
    so = (o_nib * 0x00204081) & 0x01010101
    return (sp | (so << 1)) & 0xFFFFFFFF


def cells(p: int, o: int) -> list[int]:
    return [((p >> t) & 1) + 2 * ((o >> t) & 1) for t in range(64)]


def test_cell_word_spreads_every_nibble_pair():
    # every pair, overlapping bits included (a cell of 3, as the per-square
    # formula gives for an invalid board)
    for p in range(16):
        for o in range(16):
            w = cell_word(p, o)
            for i in range(4):
                assert (w >> (8 * i)) & 0xFF == ((p >> i) & 1) + 2 * ((o >> i) & 1)


def warp_board(p: int, o: int) -> bytes:
    words = [cell_word((p >> (4 * j)) & 0xF, (o >> (4 * j)) & 0xF) for j in range(16)]
    return b"".join(w.to_bytes(4, "little") for w in words)


def lines_board(rows: list[tuple[int, int]], stride: int) -> bytearray:
    board = bytearray(64 * stride)
    for r, (p, o) in enumerate(rows):  # thread r writes board[t * stride + r]
        for t in range(32):
            board[t * stride + r] = ((p >> t) & 1) | (((o >> t) & 1) << 1)
            board[(t + 32) * stride + r] = ((p >> (t + 32)) & 1) | (((o >> (t + 32)) & 1) << 1)
    return board


def test_boards_hold_the_cells():
    rng = np.random.default_rng(5)
    rows = []
    for _ in range(256):
        occ = int(rng.integers(0, 2 ** 63, dtype=np.int64)) | (int(rng.integers(0, 2)) << 63)
        p = occ & int(rng.integers(0, 2 ** 63, dtype=np.int64))
        rows.append((p, occ & ~p))
    lb = lines_board(rows, 256)
    for r, (p, o) in enumerate(rows):
        want = cells(p, o)
        assert list(warp_board(p, o)) == want
        assert [lb[t * 256 + r] for t in range(64)] == want


def test_board_digits_equal_the_oracle_indices(orc):
    """In the expanded mode every instance is direct: the digits of a mask's
    squares (ascending) under one of the 8 board symmetries.  Digits read
    from the warp board (sum of 3^i * board[sq_i]) plus the pattern's offset
    give, per row, the same multiset of 40 indices as the oracle for the
    5-pattern set."""
    from tests.golden.make_golden import SET5

    pos = orc.generate_positions(11, 0, 64, 10, 50)
    idx = orc.group_index(SET5, 1, pos)
    offsets = np.concatenate([[0], np.cumsum([3 ** bin(m).count("1") for m in SET5])])
    syms = _symmetries()
    for r in range(len(pos)):
        board = warp_board(int(pos[r, 0]), int(pos[r, 1]))
        cand = []
        for k, m in enumerate(SET5):
            sq = [t for t in range(64) if (m >> t) & 1]
            for perm in syms:
                cand.append(int(offsets[k]) + sum(3 ** i * board[perm[t]] for i, t in enumerate(sq)))
        assert sorted(cand) == sorted(int(v) for v in idx[r])


def _symmetries():
    """The 8 board symmetries as square permutations (rows r, columns c)."""
    out = []
    for flip_d in (False, True):
        for flip_v in (False, True):
            for flip_h in (False, True):
                perm = []
                for t in range(64):
                    r, c = divmod(t, 8)
                    if flip_d:
                        r, c = c, r
                    if flip_v:
                        r = 7 - r
                    if flip_h:
                        c = 7 - c
                    perm.append(8 * r + c)
                out.append(perm)
    return out
