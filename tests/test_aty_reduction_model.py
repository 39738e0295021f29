"""A CPU model of the A'y kernel's run reduction (cassandra_b200/csrc/fast.cu:
reduce_block_entries, warp_round, lane_chain), step for step: the entry range
cut over 32 warps, rounds of 8 entries per lane, every run end adding the
lane's part of its run to the accumulator, the segmented scan over lanes
whose runs continue from their left, and the warp records combined after the
block.  On random column-sorted entry lists (runs of one entry up to runs
spanning many warps, ranges starting off a 4-entry bound, empty warp ranges)
it checks the column sums, that every accumulator index lies in the piece's
columns, and that no two lanes write one column in one round (the kernel's
adds are plain shared-memory read-modify-writes).  Integer y values make
every sum exact.  CPU only."""
import numpy as np
import pytest

LANES = WARPS = 32
PER_LANE = 8  # kItemsPerThread


class Acc:
    def __init__(self, c0, width):
        self.c0, self.width, self.v = c0, width, {}
        self.writers = {}  # (phase id, column) -> writer

    def add(self, col, val, phase, writer):
        assert self.c0 <= col < self.c0 + self.width, (col, self.c0, self.width)
        key = (phase, col)
        assert self.writers.setdefault(key, writer) == writer, f"two writers of column {col} in {phase}"
        self.v[col] = self.v.get(col, 0) + val


def lane_chain(any_, single, cont_prev, hc, ts, carry, sink):
    """lane_chain: segmented inclusive scan (shuffle-up tree) of the open sums."""
    v = [ts[i] if any_[i] else 0 for i in range(LANES)]
    f = [any_[i] and not (single[i] and cont_prev[i]) for i in range(LANES)]
    d = 1
    while d < LANES:
        vu, fu = v[:], f[:]
        for i in range(d, LANES):
            if not f[i]:
                v[i] = v[i] + vu[i - d]
            f[i] = f[i] or fu[i - d]
        d *= 2
    x = [v[i] if f[i] else v[i] + carry for i in range(LANES)]
    for i in range(LANES):
        xprev = carry if i == 0 else x[i - 1]
        if any_[i] and not single[i] and cont_prev[i]:
            sink(i, hc[i], xprev)
    return x[LANES - 1]


def reduce_block_entries(ents, y, e_lo, e_hi, acc):
    n = e_hi - e_lo

    def cut(w):
        if w == 0:
            return e_lo
        if w == WARPS:
            return e_hi
        return max(e_lo, (e_lo + n * w // WARPS) & ~3)

    recs = []
    for warp in range(WARPS):
        w_lo, w_hi = cut(warp), cut(warp + 1)
        carry, prev_end = 0, True
        rs = w_lo & ~3
        rnd = 0
        while w_lo < w_hi and rs < w_hi:
            phase = ("round", warp, rnd)
            sums, any_, first, last, ends = [0] * LANES, [False] * LANES, [1] * LANES, [1] * LANES, [0] * LANES
            for lane in range(LANES):
                ef = rs + lane * PER_LANE
                lo, hi = max(ef, w_lo), min(ef + PER_LANE, w_hi)
                s = 0
                for e in range(lo, hi):
                    s += int(y[(ents[e] & 0xFFFC) >> 2])
                    ends[lane] |= ents[e]
                    if ents[e] & 1:
                        acc.add(ents[e] >> 16, s, phase, lane)
                        s = 0
                if lo < hi:
                    any_[lane], first[lane], last[lane] = True, ents[lo], ents[hi - 1]
                sums[lane] = s
            single = [any_[i] and not (ends[i] & 1) for i in range(LANES)]
            hc = [first[i] >> 16 for i in range(LANES)]
            cont_prev = []
            for i in range(LANES):
                fv = max(rs + i * PER_LANE, w_lo)
                prev_closed = (not prev_end) if i == 0 else not (last[i - 1] & 1)
                cont_prev.append(any_[i] and fv > w_lo and prev_closed)
            sink_phase = ("sink", warp, rnd)
            if not any(single[i] and cont_prev[i] for i in range(LANES)):
                for i in range(LANES):
                    prev_ts = carry if i == 0 else sums[i - 1]
                    if any_[i] and not single[i] and cont_prev[i]:
                        acc.add(hc[i], prev_ts, sink_phase, i)
                carry = sums[min(31, (w_hi - 1 - rs) // PER_LANE)]
            else:
                carry = lane_chain(any_, single, cont_prev, hc, sums, carry,
                                   lambda i, col, val: acc.add(col, val, sink_phase, i))
            prev_end = (last[31] & 1) != 0
            rs += LANES * PER_LANE
            rnd += 1
        if w_lo < w_hi:
            ef, el = ents[w_lo], ents[w_hi - 1]
            recs.append((True, w_lo > e_lo and not (ents[w_lo - 1] & 1), ((ef ^ el) >> 16) == 0 and not (el & 1),
                         ef >> 16, carry))
        else:
            recs.append((False, False, False, 0, carry))
    lane_chain([r[0] for r in recs], [r[2] for r in recs], [r[1] for r in recs], [r[3] for r in recs],
               [r[4] for r in recs], 0, lambda i, col, val: acc.add(col, val, ("records",), i))


def _case(rng, mode):
    c0 = int(rng.integers(0, 3)) * 8192
    width = int(rng.integers(1, 200))
    runs = []
    for c in range(width):
        if rng.random() < 0.3:
            continue  # a column without entries in this block
        if mode == 0:
            ln = int(rng.integers(1, 4))
        elif mode == 1:
            ln = int(rng.geometric(1 / 6))
        elif mode == 2:
            ln = int(rng.choice([1, 2, 2500])) if rng.random() < 0.1 else int(rng.integers(1, 10))
        else:
            ln = int(rng.integers(1, 400))
        runs.append((c0 + c, ln))
    pre = int(rng.integers(0, 7))  # the range need not start on a 4-entry bound
    ents = [(0x7FFF << 16) | 1] * pre
    for col, ln in runs:
        rows = np.sort(rng.integers(0, 16384, ln))
        ents += [(col << 16) | (int(r) << 2) | (1 if i == ln - 1 else 0) for i, r in enumerate(rows)]
    e_lo, e_hi = pre, len(ents)
    ents += [(0x7FFF << 16) | 1] * 5
    return ents, c0, width, e_lo, e_hi


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_model_sums_columns_with_one_writer_per_round(mode):
    rng = np.random.default_rng(100 + mode)
    y = rng.integers(-5, 6, 16384)
    for _ in range(12):
        ents, c0, width, e_lo, e_hi = _case(rng, mode)
        acc = Acc(c0, width)
        if e_lo < e_hi:
            reduce_block_entries(ents, y, e_lo, e_hi, acc)
        want = {}
        for e in ents[e_lo:e_hi]:
            want[e >> 16] = want.get(e >> 16, 0) + int(y[(e & 0xFFFC) >> 2])
        assert set(acc.v) <= set(want)
        for col, val in want.items():
            assert acc.v.get(col, 0) == val, (mode, col)


def test_model_single_column_spanning_every_warp():
    """One run over the whole range: no run ends before the last entry, every
    lane and warp continues it; the records carry it to the last warp."""
    y = np.arange(16384) % 7 - 3
    ln = 9000
    rows = np.arange(ln) % 16384
    ents = [(5 << 16) | (int(r) << 2) | (1 if i == ln - 1 else 0) for i, r in enumerate(rows)] + [1] * 4
    acc = Acc(0, 8)
    reduce_block_entries(ents, y, 0, ln, acc)
    assert acc.v == {5: int(np.sum(y[rows]))}
