"""A CPU model of the blocked layout's per-group sort (cassandra_b200/csrc/
fast.cu: sort_pass, fast_sort_kernel), step for step: two stable 8-bit
passes over (column << 16 | row << 2) items, each in tiles of 4096 -- every
warp ranks its 512 items by digit in item order (32 lanes per step), the
warps' per-digit counts become offsets, the tile is scattered digit by digit
into a buffer and written out from there; the first pass counts the final
pass's digits while it writes; the final pass writes G32's round order
(round_phys) and sets the end flags, holding back the last entry of each
digit in a tile until the digit's next tile (or the pass's end) shows
whether the column continues.

On skewed random columns (one column only, 16-bit columns, groups of one to
two tiles and ragged last tiles) it checks that every buffer slot and output
position is written exactly once and in range, and that the result equals a
stable sort by column with a flag on the last entry of every column, stored
in round order (a partial block's last round only partly filled).  CPU only."""
import numpy as np
import pytest

THREADS, PER = 256, 16          # kSortThreads, kSortPerThread
TILE = THREADS * PER            # kSortTile
WARPS, WITEMS = THREADS // 32, 32 * PER


def round_phys(i: int) -> int:
    """G32's place of sorted position i (fast.cuh: round_phys)."""
    return (i & ~1023) | ((i & 0x1C) << 5) | ((i & 0x3E0) >> 3) | (i & 3)


def sort_pass(items, shift: int, final: bool, counts):
    n = len(items)
    room = (n + 1023) & ~1023  # the segment's rounds (a group's last round may be partial)
    out = np.zeros(room, dtype=np.int64)
    written = np.zeros(room, dtype=np.int64)
    base = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
    running = np.zeros(256, np.int64)
    hist2 = np.zeros(256, np.int64)
    pend_pos = np.full(256, -1, np.int64)
    pend_col = np.zeros(256, np.int64)
    for t0 in range(0, n, TILE):
        # 1. rank: warp w's items t0 + 512 w + 32 k + lane, in item order
        wcnt = np.zeros((WARPS, 256), np.int64)
        ranked = []
        for w in range(WARPS):
            for k in range(PER):
                step = {}
                for lane in range(32):
                    e = t0 + w * WITEMS + 32 * k + lane
                    if e < n:
                        it = int(items[e])
                        d = (it >> shift) & 255
                        r = step.get(d, 0)  # popc(peers & lanes below)
                        ranked.append((w, it, wcnt[w][d] + r))
                        step[d] = r + 1
                for d, c in step.items():  # the leader's update
                    wcnt[w][d] += c
        # 2. each warp's offset inside the tile's run of a digit
        tcount = wcnt.sum(axis=0)
        off = np.zeros_like(wcnt)
        off[1:] = np.cumsum(wcnt, axis=0)[:-1]
        tbase = np.concatenate([[0], np.cumsum(tcount)[:-1]])
        # 3. the buffer, digit by digit
        buf = np.full(TILE, -1, np.int64)
        for w, it, r in ranked:
            d = (it >> shift) & 255
            slot = tbase[d] + off[w][d] + r
            assert buf[slot] == -1
            buf[slot] = it
        tn = min(TILE, n - t0)
        assert (buf[:tn] >= 0).all() and (buf[tn:] == -1).all()
        # 4. out
        for j in range(tn):
            it = int(buf[j])
            d = (it >> shift) & 255
            pos = base[d] + running[d] + j - tbase[d]
            assert 0 <= pos < n
            if final:
                last_in_tile = j + 1 == tbase[d] + tcount[d]
                if not last_in_tile and (int(buf[j + 1]) >> 16) != (it >> 16):
                    it |= 1
                pos = round_phys(pos)
                assert 0 <= pos < room
            else:
                hist2[it >> 24] += 1
            out[pos] = it
            written[pos] += 1
        if final:
            for d in range(256):
                if tcount[d] > 0:
                    if pend_pos[d] >= 0 and (int(buf[tbase[d]]) >> 16) != pend_col[d]:
                        out[round_phys(pend_pos[d])] |= 1
                    pend_pos[d] = base[d] + running[d] + tcount[d] - 1
                    pend_col[d] = int(buf[tbase[d] + tcount[d] - 1]) >> 16
        running += tcount
    if final:
        for d in range(256):
            if pend_pos[d] >= 0:
                out[round_phys(pend_pos[d])] |= 1
    assert written.sum() == n and written.max() == 1
    if not final:
        assert (written[:n] == 1).all()
    return out, hist2


@pytest.mark.parametrize("rows,slots,cols,skew", [
    (1024, 8, 59049, 1.0),   # two full tiles, 3^10 columns
    (1024, 5, 65535, 0.7),   # a ragged last tile, 16-bit columns
    (1024, 3, 2187, 2.0),    # one ragged tile
    (1024, 4, 1, 1.0),       # one column: one run over every tile
    (777, 3, 19683, 1.2),    # a partial block: n not a multiple of 8 or of a round
])
def test_sort_passes_equal_a_stable_column_sort(rows, slots, cols, skew):
    rng = np.random.default_rng(rows * slots + cols)
    n = rows * slots
    col = (rng.zipf(1 + skew, size=n) * 7919) % cols
    items = (col.astype(np.int64) << 16) | ((np.arange(n) // slots) << 2)
    mid, hist2 = sort_pass(items, 16, False, np.bincount((items >> 16) & 255, minlength=256))
    out, _ = sort_pass(mid[:n], 24, True, hist2)
    want = items[np.argsort(col, kind="stable")]
    ends = np.ones(n, dtype=np.int64)
    ends[:-1] = (want[1:] >> 16) != (want[:-1] >> 16)
    got = out[[round_phys(i) for i in range(n)]]
    np.testing.assert_array_equal(got, want | ends)
