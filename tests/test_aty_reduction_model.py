"""A CPU model of the A'y kernel's run reduction (cassandra_b200/csrc/fast.cu:
reduce_block, lane_entries, lane_chain, and the piece table aty_item builds),
step for step: the column-sorted entries stored in G32 rounds (round_phys:
lane L's 32 consecutive entries spread over 8 rows of 16-byte words), the
pieces' entry ranges cut into virtual rounds that 32 warps split into
stretches, 32 entries per lane and round with the entries outside a piece's
range masked, every run end adding the lane's part of its run to the
accumulator, the segmented scan over lanes whose runs continue from their
left, and the warp records combined after the block.  The FP64 items use
the stretch reduction instead (reduce_stretch, stretch_step): each piece's
range cut into 32 stretches of whole 4-entry words, 16 entries per lane and
step, read through round_phys; it is modelled the same way.

On random blocks (several pieces in different groups, runs of one entry up
to runs spanning many warps, piece ranges starting and ending anywhere in a
round, pieces without entries, more warps than rounds) it checks the column
sums, that every load lies in the piece's group and returns the entry the
sorted order puts there, that every accumulator index lies in its piece's
columns, that no two lanes write one column in one step (the kernel's adds
are plain shared-memory read-modify-writes), and that every virtual round
holds an entry of its piece.  Integer y values make every sum exact.
CPU only."""
import numpy as np
import pytest

LANES = WARPS = 32
ROUND = 1024
RUN = 32  # kLaneRun


def round_phys(i: int) -> int:
    """G32's place of sorted position i (fast.cuh: round_phys)."""
    return (i & ~(ROUND - 1)) | ((i & 0x1C) << 5) | ((i & 0x3E0) >> 3) | (i & 3)


def test_round_phys_is_a_permutation_of_each_round():
    got = sorted(round_phys(i) for i in range(3 * ROUND))
    assert got == list(range(3 * ROUND))
    # lane L's slot s sits in word 32 q + L (q = s // 4) of the round, entry s % 4
    for lane in range(LANES):
        for s in range(RUN):
            assert round_phys(RUN * lane + s) == 4 * (32 * (s // 4) + lane) + s % 4


class Acc:
    def __init__(self, width):
        self.width, self.v = width, {}
        self.writers = {}  # (step id, index) -> writer

    def add(self, idx, val, step, writer, lo_idx, hi_idx):
        assert 0 <= idx < self.width and lo_idx <= idx < hi_idx, (idx, lo_idx, hi_idx)
        key = (step, idx)
        assert self.writers.setdefault(key, writer) == writer, f"two writers of {idx} in {step}"
        self.v[idx] = self.v.get(idx, 0) + val


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


def reduce_block(g32, pieces, y, acc):
    """pieces: (lo, hi, acc_off, seg, seg_end, col_lo, col_hi) per piece;
    g32 holds every group in round order."""
    round0 = [0]
    for lo, hi, *_ in pieces:
        round0.append(round0[-1] + ((hi - 1) // ROUND - lo // ROUND + 1 if lo < hi else 0))
    nrounds = round0[-1]
    recs = []
    for warp in range(WARPS):
        vr0, vr1 = nrounds * warp // WARPS, nrounds * (warp + 1) // WARPS
        carry, prev_end, w_end, w_cp, w_fc = 0, True, False, False, 0
        k = 0
        while k < len(pieces) and round0[k + 1] <= vr0:
            k += 1
        for vr in range(vr0, vr1):
            if vr >= round0[k + 1]:
                while vr >= round0[k + 1]:
                    k += 1
                carry, prev_end = 0, True
            lo, hi, off, seg, seg_end, col_lo, col_hi = pieces[k]
            rbase = (lo // ROUND + (vr - round0[k])) * ROUND
            assert seg <= rbase and rbase + ROUND <= seg_end  # the round (and its prefetch) lies in the group
            step = ("round", warp, vr)
            sums, any_, first, last, eor, f = [0] * LANES, [False] * LANES, [1] * LANES, [1] * LANES, \
                [0] * LANES, [0] * LANES

            def sink_at(ph):
                return lambda i, col, val: acc.add(off + col, val, ph, i, col_lo, col_hi)

            for lane in range(LANES):
                lb = rbase + RUN * lane
                k0 = min(lo - lb, RUN) if lo > lb else 0
                k1 = min(hi - lb, RUN) if hi > lb else 0
                s_sum, o = 0, 0
                for s in range(RUN):
                    word = rbase + 4 * (32 * (s // 4) + lane) + s % 4  # src + 32 q, entry s % 4
                    e = g32[word]
                    if k0 <= s < k1:
                        assert e == g32[round_phys(lb + s)]
                        s_sum += int(y[(e & 0xFFFC) >> 2])
                        o |= e
                        if e & 1:
                            acc.add(off + (e >> 16), s_sum, step + ("end", s), lane, col_lo, col_hi)
                            s_sum = 0
                        if s == k0:
                            first[lane] = e
                        last[lane] = e
                any_[lane], sums[lane], eor[lane], f[lane] = k0 < k1, s_sum, o, lb + k0
            assert any(any_), "a virtual round without an entry of its piece"
            single = [any_[i] and not (eor[i] & 1) for i in range(LANES)]
            hc = [first[i] >> 16 for i in range(LANES)]
            cont_prev = []
            for i in range(LANES):
                if i == 0:
                    prev_open = vr != vr0 and not prev_end
                else:
                    prev_open = not (last[i - 1] & 1)
                cont_prev.append(any_[i] and f[i] > lo and prev_open)
            lastl = max(i for i in range(LANES) if any_[i])
            if not any(single[i] and cont_prev[i] for i in range(LANES)):
                for i in range(LANES):
                    prev_ts = carry if i == 0 else sums[i - 1]
                    if any_[i] and not single[i] and cont_prev[i]:
                        sink_at(step + ("sink",))(i, hc[i], prev_ts)
                carry = sums[lastl]
            else:
                carry = lane_chain(any_, single, cont_prev, hc, sums, carry, sink_at(step + ("sink",)))
            prev_end = (last[lastl] & 1) != 0
            if vr == vr0:
                fl = min(i for i in range(LANES) if any_[i])
                w_fc = off + (first[fl] >> 16)
                f0 = f[fl]
                w_cp = f0 > lo and not (g32[round_phys(f0 - 1)] & 1)
            w_end = w_end or any(any_[i] and not single[i] for i in range(LANES))
        recs.append((vr0 < vr1, w_cp, not w_end, w_fc, carry))
    lane_chain([r[0] for r in recs], [r[2] for r in recs], [r[1] for r in recs], [r[3] for r in recs],
               [r[4] for r in recs], 0, lambda i, idx, val: acc.add(idx, val, ("records",), i, 0, acc.width))


def _runs(rng, mode, width):
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
        runs.append((c, ln))
    return runs


def _block(rng, mode, npieces):
    """Groups of sorted entries (one per piece, each starting on a round and
    padded to whole rounds, stored in round order), a piece range inside each
    group starting and ending on column boundaries (the columns before and
    after belong to other splits), and the accumulator width."""
    logical, pieces, acc_w = [], [], 0
    for _ in range(npieces):
        seg = len(logical)
        c0 = int(rng.integers(0, 3)) * 8192
        before, width, after = int(rng.integers(0, 30)), int(rng.integers(1, 200)), int(rng.integers(0, 30))
        flat, lo, hi = [], None, None
        for c, ln in _runs(rng, mode, before + width + after):
            if lo is None and c >= before:
                lo = seg + len(flat)
            if hi is None and c >= before + width:
                hi = seg + len(flat)
            rows = np.sort(rng.integers(0, 16384, ln))
            flat += [((c0 + c) << 16) | (int(r) << 2) | (1 if i == ln - 1 else 0) for i, r in enumerate(rows)]
        lo = seg + len(flat) if lo is None else lo
        hi = seg + len(flat) if hi is None else hi
        logical += flat + [0xFFFFFFFE] * ((-len(flat)) % ROUND)  # group padding (never in a range)
        if not flat:
            logical += [0xFFFFFFFE] * ROUND
        pieces.append((lo, hi, acc_w - (c0 + before), seg, len(logical), acc_w, acc_w + width))
        acc_w += width
    g32 = [0] * len(logical)
    for i, e in enumerate(logical):
        g32[round_phys(i)] = e
    return g32, logical, pieces, acc_w


def _expect(logical, pieces, y):
    want = {}
    for lo, hi, off, *_ in pieces:
        for e in logical[lo:hi]:
            want[off + (e >> 16)] = want.get(off + (e >> 16), 0) + int(y[(e & 0xFFFC) >> 2])
    return want


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_model_sums_columns_with_one_writer_per_step(mode):
    rng = np.random.default_rng(100 + mode)
    y = rng.integers(-5, 6, 16384)
    for trial in range(8):
        g32, logical, pieces, width = _block(rng, mode, 1 + trial % 4)
        acc = Acc(width)
        reduce_block(g32, pieces, y, acc)
        want = _expect(logical, pieces, y)
        assert set(acc.v) <= set(want)
        for col, val in want.items():
            assert acc.v.get(col, 0) == val, (mode, trial, col)


def test_model_single_column_spanning_every_warp():
    """One run over many rounds: no run ends before its last entry, every
    lane and warp continues it; the records carry it to the last warp."""
    y = np.arange(16384) % 7 - 3
    ln = 40_000
    rows = np.arange(ln) % 16384
    logical = [(5 << 16) | (int(r) << 2) | (1 if i == ln - 1 else 0) for i, r in enumerate(rows)]
    logical += [0xFFFFFFFE] * ((-ln) % ROUND)
    g32 = [0] * len(logical)
    for i, e in enumerate(logical):
        g32[round_phys(i)] = e
    acc = Acc(8)
    reduce_block(g32, [(0, ln, 0, 0, len(logical), 0, 8)], y, acc)
    assert acc.v == {5: int(np.sum(y[rows]))}


def test_model_few_rounds_and_empty_pieces():
    """Fewer rounds than warps (most warps idle), a piece without entries
    between two others, and ranges that start and end inside one round."""
    rng = np.random.default_rng(7)
    y = rng.integers(-5, 6, 16384)
    logical = []
    pieces = []
    for lo_off, n, width in ((37, 50, 20), (0, 0, 5), (700, 900, 40)):
        seg = len(logical)
        ents = []
        per = max(1, n // width) if n else 0
        left = n
        for c in range(width):
            ln = min(left, per if c < width - 1 else left)
            rows = np.sort(rng.integers(0, 16384, ln))
            ents += [((100 + c) << 16) | (int(r) << 2) | (1 if i == ln - 1 else 0) for i, r in enumerate(rows)]
            left -= ln
        pre = [(99 << 16) | 1] * lo_off
        flat = pre + ents
        logical += flat + [0xFFFFFFFE] * ((-len(flat)) % ROUND or (ROUND if not flat else 0))
        aw = sum(p[6] - p[5] for p in pieces)
        pieces.append((seg + lo_off, seg + lo_off + len(ents), aw - 100, seg, len(logical), aw, aw + width))
    g32 = [0] * len(logical)
    for i, e in enumerate(logical):
        g32[round_phys(i)] = e
    acc = Acc(sum(p[6] - p[5] for p in pieces))
    reduce_block(g32, pieces, y, acc)
    want = _expect(logical, pieces, y)
    for col, val in want.items():
        assert acc.v.get(col, 0) == val


STEP = 16  # kStretchRun


def reduce_stretch(g32, y, e_lo, e_hi, acc, off, col_lo, col_hi):
    """reduce_stretch / stretch_step over sorted positions [e_lo, e_hi) of a
    group stored in round order."""
    n = e_hi - e_lo

    def cut(w):
        if w == 0:
            return e_lo
        if w == WARPS:
            return e_hi
        return max(e_lo, (e_lo + n * w // WARPS) & ~3)

    def at(e):
        return g32[round_phys(e)]

    recs = []
    for warp in range(WARPS):
        w_lo, w_hi = cut(warp), cut(warp + 1)
        carry, prev_end = 0, True
        rs, rnd = w_lo & ~3, 0
        while w_lo < w_hi and rs < w_hi:
            step = ("step", warp, rnd)
            sums, any_, first, last, ends = [0] * LANES, [False] * LANES, [1] * LANES, [1] * LANES, [0] * LANES
            for lane in range(LANES):
                ef = rs + lane * STEP
                full = ef >= w_lo and ef + STEP <= w_hi
                if full:  # STEP / 4 16-byte words: round_phys of ef, ef + 4, ..., 4 entries each
                    words = [g32[round_phys(ef + 4 * q) + j] for q in range(STEP // 4) for j in range(4)]
                    assert words == [at(e) for e in range(ef, ef + STEP)]
                lo, hi = max(ef, w_lo), min(ef + STEP, w_hi)
                s = 0
                for e in range(lo, hi):
                    v = at(e)
                    s += int(y[(v & 0xFFFC) >> 2])
                    ends[lane] |= v
                    if v & 1:
                        acc.add(off + (v >> 16), s, step + ("end", e - ef), lane, col_lo, col_hi)
                        s = 0
                if lo < hi:
                    any_[lane], first[lane], last[lane] = True, at(lo), at(hi - 1)
                sums[lane] = s
            single = [any_[i] and not (ends[i] & 1) for i in range(LANES)]
            hc = [first[i] >> 16 for i in range(LANES)]
            cont_prev = []
            for i in range(LANES):
                fv = max(rs + i * STEP, w_lo)
                prev_open = (not prev_end) if i == 0 else not (last[i - 1] & 1)
                cont_prev.append(any_[i] and fv > w_lo and prev_open)
            sink = lambda i, col, val: acc.add(off + col, val, step + ("sink",), i, col_lo, col_hi)  # noqa: E731
            if not any(single[i] and cont_prev[i] for i in range(LANES)):
                for i in range(LANES):
                    prev_ts = carry if i == 0 else sums[i - 1]
                    if any_[i] and not single[i] and cont_prev[i]:
                        sink(i, hc[i], prev_ts)
                carry = sums[min(31, (w_hi - 1 - rs) // STEP)]
            else:
                carry = lane_chain(any_, single, cont_prev, hc, sums, carry, sink)
            prev_end = (last[31] & 1) != 0
            rs += LANES * STEP
            rnd += 1
        if w_lo < w_hi:
            ef, el = at(w_lo), at(w_hi - 1)
            recs.append((True, w_lo > e_lo and not (at(w_lo - 1) & 1), ((ef ^ el) >> 16) == 0 and not (el & 1),
                         ef >> 16, carry))
        else:
            recs.append((False, False, False, 0, carry))
    lane_chain([r[0] for r in recs], [r[2] for r in recs], [r[1] for r in recs], [r[3] for r in recs],
               [r[4] for r in recs], 0,
               lambda i, col, val: acc.add(off + col, val, ("records",), i, col_lo, col_hi))


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_stretch_model_sums_columns(mode):
    rng = np.random.default_rng(200 + mode)
    y = rng.integers(-5, 6, 16384)
    for trial in range(6):
        g32, logical, pieces, width = _block(rng, mode, 1 + trial % 3)
        acc = Acc(width)
        for lo, hi, off, seg, seg_end, col_lo, col_hi in pieces:
            if lo < hi:
                reduce_stretch(g32, y, lo, hi, acc, off, col_lo, col_hi)
        want = _expect(logical, pieces, y)
        assert set(acc.v) <= set(want)
        for col, val in want.items():
            assert acc.v.get(col, 0) == val, (mode, trial, col)
