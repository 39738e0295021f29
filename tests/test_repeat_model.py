"""A CPU model of the repeats' share of diag(A'A) on the blocked layout
(cassandra_b200/csrc/fast.cu: fast_repeat_kernel), step for step: a warp
takes a stretch of 16 rounds of a sorted group stored in round order
(round_phys); per round each lane reads its 32 consecutive sorted entries
from eight 16-byte words 512 bytes apart, counts the equal entries ending its
run, takes the entry before its run and that count from the lane before it
(lane 0: from lane 31 of the previous round, or walked back in G32 at the
stretch's start), counts copies of each (column, row) along its run and adds
2 (1 + ... + (m - 1)) per column, once per run of that column.

Checked against sum over rows of m (m - 1) per column on groups with
repeats of up to 8 copies (runs that cross lanes, rounds and stretches), a
partial last round and one-column groups.  CPU only."""
import numpy as np
import pytest

ROUND, LANE_RUN, STRETCH_ROUNDS = 1024, 32, 16


def round_phys(i: int) -> int:
    return (i & ~1023) | ((i & 0x1C) << 5) | ((i & 0x3E0) >> 3) | (i & 3)


def repeat_model(g32: np.ndarray, n: int, ncols: int, stretches: int) -> np.ndarray:
    diag = np.zeros(ncols, np.int64)
    touched = np.zeros(len(g32), np.int64)
    for st in range(stretches):
        r_begin = st * STRETCH_ROUNDS * ROUND
        if r_begin >= n:
            continue
        r_end = min(n, r_begin + STRETCH_ROUNDS * ROUND)
        carry_last, carry_tail = 0, 0
        if r_begin > 0:
            carry_last = int(g32[round_phys(r_begin - 1)])
            carry_tail = 1
            while carry_tail < r_begin and (int(g32[round_phys(r_begin - 1 - carry_tail)]) >> 2) == (carry_last >> 2):
                carry_tail += 1
        for r0 in range(r_begin, r_end, ROUND):
            runs, tails, lasts, cnts = [], [], [], []
            for lane in range(32):
                lb = r0 + LANE_RUN * lane
                cnt = max(0, min(LANE_RUN, r_end - lb))
                e = [0] * LANE_RUN
                for q in range(LANE_RUN // 4):  # word q of the lane: uint4 index 32 q + lane of the round
                    if 4 * q < cnt:
                        w0 = r0 + 4 * (32 * q + lane)
                        assert w0 + 4 <= len(g32)
                        for j in range(4):
                            e[4 * q + j] = int(g32[w0 + j])
                            touched[w0 + j] += 1
                tail, last = 0, 0
                for k in range(cnt):
                    tail = tail + 1 if k > 0 and (e[k] >> 2) == (e[k - 1] >> 2) else 1
                    last = e[k]
                runs.append(e), tails.append(tail), lasts.append(last), cnts.append(cnt)
            for lane in range(32):
                before, m = (carry_last, carry_tail) if lane == 0 else (lasts[lane - 1], tails[lane - 1])
                e, cnt = runs[lane], cnts[lane]
                acc, acc_col = 0, (e[0] >> 16 if cnt else 0)
                for k in range(cnt):
                    col = e[k] >> 16
                    if col != acc_col:
                        diag[acc_col] += acc
                        acc, acc_col = 0, col
                    if m > 0 and (e[k] >> 2) == (before >> 2):
                        acc += 2 * m
                        m += 1
                    else:
                        m = 1
                    before = e[k]
                diag[acc_col] += acc
            carry_last, carry_tail = lasts[31], tails[31]
    return diag, touched


@pytest.mark.parametrize("rows,slots,ncols,seed", [
    (16384, 8, 400, 1),     # 128 rounds: 8 full stretches, runs of 8 copies across lanes and rounds
    (5000, 8, 3, 2),        # three columns: long column runs, a partial last round
    (777, 5, 1, 3),         # one column
    (3001, 3, 20000, 4),    # few repeats
])
def test_repeat_model_equals_sum_of_m_squared_minus_m(rows, slots, ncols, seed):
    rng = np.random.default_rng(seed)
    # every row holds `slots` entries; heavy repeats: a row often takes one
    # column for several of its slots
    col = np.empty((rows, slots), np.int64)
    for r in range(rows):
        k = 0
        while k < slots:
            m = int(rng.integers(1, slots - k + 1))
            col[r, k:k + m] = rng.integers(0, ncols)
            k += m
    n = rows * slots
    row = np.repeat(np.arange(rows), slots)
    items = (col.reshape(-1) << 16) | (row << 2)
    items = np.sort(items, kind="stable")  # column-major, rows ascending (the sort's order)
    ends = np.ones(n, np.int64)
    ends[:-1] = (items[1:] >> 16) != (items[:-1] >> 16)
    room = (n + ROUND - 1) // ROUND * ROUND
    g32 = np.full(room, 0xFFFFFFFF, np.int64)  # the last round's unused slots hold anything
    g32[[round_phys(i) for i in range(n)]] = items | ends
    stretches = (16384 * slots + STRETCH_ROUNDS * ROUND - 1) // (STRETCH_ROUNDS * ROUND)
    got, touched = repeat_model(g32, n, ncols, stretches)
    want = np.zeros(ncols, np.int64)
    for c_r in np.unique(items >> 2):
        m = int((items >> 2 == c_r).sum())
        want[c_r >> 14] += m * (m - 1)
    np.testing.assert_array_equal(got, want)
    assert (touched[[round_phys(i) for i in range(n)]] == 1).all()  # every entry read once
    assert want.sum() > 0 or ncols > 1000
