"""CPU model of the count kernel's filtered DFS step, checked against the oracle.

The GPU kernel's default count step (``NQB_STEP4`` in
n_queens_b200/csrc/dfs_kernel.cuh, with ``load_task`` / ``settle_level`` /
``alive_columns``) drops children that would leave the next row without a
free column and counts children on row N-2 without entering them.  This file
restates that step operation by operation in 32-bit numpy arithmetic, one
array element per lane (no donation, which moves stack entries between lanes
but changes no arithmetic), and checks three things on the CPU:

* per-task counts equal the oracle's restatement of the reference recursion
  (src/n_queens.cpp:8-21) on whole-board prefix lists and on arbitrary 32-bit
  (cols, left, right) triples, off-board bits included;
* the deepest stack a lane ever holds is at most N-3-popc(cols) slots, the
  per-task need the launch reserves for the filtered step;
* an idle lane (no untried column, empty stack) is left unchanged by further
  steps, which is what lets a warp keep stepping while some lanes wait.

The dihedral kernels' filtered step (``NQB_STEP_DIH4``: dead children dropped,
rows N-2 and N-1 still stepped under the class rules) is restated the same way
and checked against the oracle's weighted per-task counts of the dihedral
decomposition (oracle/dihedral_oracle.c) and the whole-board totals.
"""
import numpy as np
import pytest

import oracle

def popc(x):
    return np.bitwise_count(x).astype(np.uint32)


def sar1(x):
    """shr.s32 x, x, 1 (arithmetic, as the reference's int arithmetic)."""
    return (x.view(np.int32) >> 1).view(np.uint32)


def shiftamt(x):
    """bfind.shiftamt.u32: 31 - index of the highest set bit, 0xffffffff for 0."""
    s = x.copy()
    for k in (1, 2, 4, 8, 16):
        s |= s >> np.uint32(k)
    hi = popc(s).astype(np.int64) - 1
    return np.where(x == 0, np.uint32(0xFFFFFFFF), (31 - hi).astype(np.uint32))


def shr_clamp(a, n):
    """shr.b32 with the shift amount clamped to 32 (a shift of 32 or more gives 0)."""
    n64 = n.astype(np.int64)
    return np.where(n64 >= 32, np.uint32(0), (np.uint64(a) >> np.minimum(n64, 31).astype(np.uint64)).astype(np.uint32))


def alive_columns(cols, ld, rd, avail):
    """alive_columns(): the untried columns whose child leaves the next row a free column."""
    f0 = ~(cols | ld | sar1(rd))
    lo = f0 & (np.uint32(0) - f0)
    hi = 31 - shiftamt(f0).astype(np.int64)
    above = np.uint32(0) - (lo << np.uint32(2))
    below = np.where(hi >= 2, (np.uint64(0xFFFFFFFF) >> (33 - np.maximum(hi, 2)).astype(np.uint64)).astype(np.uint32),
                     np.uint32(0))
    return np.where(f0 == 0, np.uint32(0), avail & (above | below))


def load_tasks(N, c, l, r):
    """load_task<4>: lane registers and the completions credited at load time."""
    last = np.uint32(0xFFFFFFFF if N >= 32 else (1 << N) - 1)
    bad = (c & ~last) != 0
    done = (c == last) & ~bad
    cols = c | ~last
    ld = l << np.uint32(1)
    rd = r.copy()
    avail = ~(cols | l | r)
    avail = np.where(bad | done, np.uint32(0), avail)
    credit = done.astype(np.uint64)
    # settle_level: rows N-1 and N-2 complete at load time.
    row = popc(cols).astype(np.int64) - (32 - N)
    last_row = (row >= N - 1) & (avail != 0)
    credit += np.where(last_row, popc(avail), 0).astype(np.uint64)
    avail = np.where(last_row, np.uint32(0), avail)
    avail = np.where(avail != 0, alive_columns(cols, ld, rd, avail), avail)
    n2 = (row == N - 2) & (avail != 0)
    credit += np.where(n2, popc(avail), 0).astype(np.uint64)
    avail = np.where(n2, np.uint32(0), avail)
    return cols, ld, rd, avail, credit


class Lanes:
    """Lane registers (cols, ld in lane form, rd, avail), per-lane stacks and counters."""

    def __init__(self, N, c, l, r):
        c, l, r = (np.ascontiguousarray(a, np.uint32) for a in (c, l, r))
        self.n = c.size
        self.cols, self.ld, self.rd, self.avail, self.credit = load_tasks(N, c, l, r)
        self.stack = np.zeros((self.n, N + 2, 4), np.uint32)
        self.sp = np.zeros(self.n, np.int64)          # slots in use (sp - bot in the kernel)
        self.deepest = np.zeros(self.n, np.int64)
        self.cnt = np.zeros(self.n, np.uint64)

    def step(self):
        """One NQB_STEP4 on every lane, operation by operation (%8 = 1, %9 = 2, %10 = -1, %13 = -4, %14 = 30)."""
        one, two, mone, m4 = np.uint32(1), np.uint32(2), np.uint32(0xFFFFFFFF), np.uint32(0xFFFFFFFC)
        cols, ld, rd, avail = self.cols, self.ld, self.rd, self.avail
        t = avail * mone
        bit = t & avail
        pb = bit != 0
        nc = bit * one + cols
        nl = bit * two + ld
        nr = sar1(rd | bit)
        na = ~(nc | nl | nr)
        xl = nl * two
        xr = sar1(nr)
        f0 = ~(nc | xl | xr)
        lo = (np.uint32(0) - f0) & f0
        ma = lo * m4
        mb = shr_clamp(np.uint32(0x3FFFFFFF), shiftamt(f0))
        pc = popc(nc)
        pg = (pc != 30) & pb
        p2 = (pc == 30) & pb
        naf = na & (ma | mb)
        pd = (naf != 0) & pg
        self.cnt += np.where(p2, popc(naf), 0).astype(np.uint64)
        avail = avail ^ bit
        pk = (avail != 0) | pd
        pp = (avail != 0) & pd
        # push the parent's remaining columns, then move to the child
        lanes = np.arange(self.n)
        idx = lanes[pp]
        self.stack[idx, self.sp[idx]] = np.stack([cols[idx], ld[idx], rd[idx], avail[idx]], axis=1)
        self.sp[idx] += 1
        self.deepest = np.maximum(self.deepest, self.sp)
        cols = np.where(pd, nc, cols)
        ld = np.where(pd, xl, ld)
        rd = np.where(pd, nr, rd)
        avail = np.where(pd, naf, avail)
        pq = (self.sp != 0) & ~pk
        idx = lanes[pq]
        self.sp[idx] -= 1
        top = self.stack[idx, self.sp[idx]]
        cols[idx], ld[idx], rd[idx], avail[idx] = top[:, 0], top[:, 1], top[:, 2], top[:, 3]
        self.cols, self.ld, self.rd, self.avail = cols, ld, rd, avail

    def run(self, max_steps=10_000_000):
        for _ in range(max_steps):
            if not self.avail.any():
                break
            self.step()
        else:
            raise AssertionError("lanes did not finish")
        # A lane whose level runs out pops in the same step, so avail = 0 means an empty stack.
        assert not self.sp.any(), "a lane went idle with stacked levels"
        return self.cnt + self.credit


def run_lanes(N, c, l, r):
    """Steps every lane to completion; returns per-lane counts and the deepest stack each lane held."""
    lanes = Lanes(N, c, l, r)
    return lanes.run(), lanes.deepest


def oracle_counts(N, c, l, r):
    return oracle.count_tasks(N, c, l, r)


def need_slots(N, c):
    """The launch's per-task stack need for the filtered step (launch.h stack_need)."""
    return np.maximum(1, N - 3 - popc(np.ascontiguousarray(c, np.uint32)).astype(np.int64))


@pytest.mark.parametrize("N,k", [(4, 1), (5, 2), (6, 2), (7, 3), (8, 2), (9, 3), (10, 3), (11, 4), (12, 5)])
def test_whole_board_prefixes(N, k):
    c, l, r = oracle.expand(N, k)
    got, deepest = run_lanes(N, c, l, r)
    np.testing.assert_array_equal(got, oracle_counts(N, c, l, r))
    assert (deepest <= need_slots(N, c)).all()


@pytest.mark.parametrize("N,n,sparse", [(8, 3000, False), (10, 3000, False), (12, 1500, False), (13, 1500, False),
                                        (10, 3000, True)])
def test_arbitrary_32bit_tasks(N, n, sparse):
    rng = np.random.default_rng(1000 + N + 100 * sparse)
    last = (1 << N) - 1

    def rand():
        return rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)

    # Partial boards with arbitrary diagonal bits (bit 31 included), a tenth with off-board columns.
    if sparse:
        c, l, r = rand() & rand(), rand() & rand(), rand() & rand()
    else:
        c = np.where(rng.random(n) < 0.5, rand() | rand(), rand() & rand())
        l, r = rand() & (rand() | rand()), rand() & (rand() | rand())
    c = np.where(rng.random(n) < 0.9, c & np.uint32(last), c)
    got, deepest = run_lanes(N, c, l, r)
    np.testing.assert_array_equal(got, oracle_counts(N, c, l, r))
    assert got.sum() > 0
    on_board = (c & ~np.uint32(last)) == 0
    assert (deepest[on_board] <= need_slots(N, c[on_board])).all()


def test_edge_rows_and_full_boards():
    # Tasks on rows N-1 and N-2, complete boards, empty boards and off-board columns.
    N = 9
    c, l, r = oracle.expand(N, N - 1)
    c2, l2, r2 = oracle.expand(N, N - 2)
    c3, l3, r3 = oracle.expand(N, N)
    extra_c = np.array([0, (1 << N) - 1, 1 << N, 0xFFFFFFFF, 0x1FF], np.uint32)
    extra_l = np.array([0, 0, 0, 0, 0xFFFFFFFF], np.uint32)
    extra_r = np.array([0, 0, 0, 0, 0x80000000], np.uint32)
    C, L, R = (np.concatenate(x) for x in ((c, c2, c3, extra_c), (l, l2, l3, extra_l), (r, r2, r3, extra_r)))
    got, _ = run_lanes(N, C, L, R)
    np.testing.assert_array_equal(got, oracle_counts(N, C, L, R))


def test_alive_columns_matches_definition():
    # A column b of the next row is dead exactly when the row after it has no free column once b is placed.
    rng = np.random.default_rng(7)
    n = 20000
    N = 12
    last = np.uint32((1 << N) - 1)
    cols = (rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32) & last) | ~last
    left = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    ld = left << np.uint32(1)
    rd = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    avail = ~(cols | left | rd)
    got = alive_columns(cols, ld, rd, avail)
    want = np.zeros(n, np.uint32)
    for b in range(32):
        m = np.uint32(1 << b)
        f_after = ~((cols | m) | ld | (m << np.uint32(1)) | sar1(rd | m))
        has = (avail & m) != 0
        want |= np.where(has & (f_after != 0), m, np.uint32(0))
    np.testing.assert_array_equal(got, want)


def test_step_formula_for_the_highest_bit_mask():
    # 0x3fffffff >> shiftamt(F0) is the set of columns at most highest(F0) - 2, and 0 for F0 = 0.
    f0 = np.concatenate([np.array([0, 1, 2, 3, 4, 0x80000000, 0xFFFFFFFF], np.uint32),
                         np.random.default_rng(3).integers(0, 1 << 32, 5000, dtype=np.uint64).astype(np.uint32)])
    got = shr_clamp(np.uint32(0x3FFFFFFF), shiftamt(f0))
    hi = 31 - shiftamt(f0).astype(np.int64)
    want = np.where((f0 != 0) & (hi >= 2), ((np.uint64(1) << np.maximum(hi - 1, 0).astype(np.uint64)) - 1), 0)
    np.testing.assert_array_equal(got, want.astype(np.uint32))


def test_idle_lanes_are_unchanged():
    N = 10
    c, l, r = oracle.expand(N, 3)
    lanes = Lanes(N, c, l, r)
    got = lanes.run()
    before = [a.copy() for a in (lanes.cols, lanes.ld, lanes.rd, lanes.avail, lanes.cnt, lanes.sp)]
    for _ in range(3):
        lanes.step()
    for a, b in zip(before, (lanes.cols, lanes.ld, lanes.rd, lanes.avail, lanes.cnt, lanes.sp)):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(got, oracle_counts(N, c, l, r))


# ---- The dihedral kernels' filtered step (NQB_STEP_DIH4) --------------------------------------------

def bfind(x):
    """bfind.u32: index of the highest set bit, 0xffffffff for 0."""
    return np.where(x == 0, np.uint32(0xFFFFFFFF), (31 - shiftamt(x).astype(np.int64)).astype(np.uint32))


class DihLanes:
    """Lanes of a dihedral kernel: the task's class rules ride in per-lane registers."""

    def __init__(self, N, c, l, r, cls, classes):
        c, l, r = (np.ascontiguousarray(a, np.uint32) for a in (c, l, r))
        cls = np.ascontiguousarray(cls, np.int64)
        tab = np.array([(min(32 - N + s, 64), lm, tb, w, wt) for (s, lm, tb, w, wt) in classes], np.uint64)
        self.side_popc = tab[cls, 0].astype(np.uint32)
        self.last_mask = tab[cls, 1].astype(np.uint32)
        self.tie_bit = tab[cls, 2].astype(np.uint32)
        self.w = tab[cls, 3].astype(np.uint32)
        self.w_tie = tab[cls, 4].astype(np.uint32)
        self.noside = np.uint32(~((1 << 0) | (1 << (N - 1))) & 0xFFFFFFFF)
        # load_task<3>: no settling; a complete board weighs the class weight.
        last = np.uint32(0xFFFFFFFF if N >= 32 else (1 << N) - 1)
        bad = (c & ~last) != 0
        done = (c == last) & ~bad
        self.cols = c | ~last
        self.ld = l << np.uint32(1)
        self.rd = r.copy()
        avail = np.where(bad | done, np.uint32(0), ~(self.cols | l | r))
        # The task's own row follows the class rules too.
        pc = popc(self.cols)
        rule = (avail != 0) & (pc > self.side_popc)
        avail = np.where(rule, avail & np.where(pc == 31, self.last_mask, self.noside), avail)
        self.avail = avail
        self.credit = np.where(done, self.w, 0).astype(np.uint64)
        self.n = c.size
        self.stack = np.zeros((self.n, N + 2, 4), np.uint32)
        self.sp = np.zeros(self.n, np.int64)
        self.deepest = np.zeros(self.n, np.int64)
        self.cnt = np.zeros(self.n, np.uint64)

    def step(self):
        """One NQB_STEP_DIH4 on every lane (%12 side popc, %13 row N-1 mask, %14 tie bit, %15/%16 weights,
        %17 ~side columns)."""
        one, two, mone, m4 = np.uint32(1), np.uint32(2), np.uint32(0xFFFFFFFF), np.uint32(0xFFFFFFFC)
        cols, ld, rd, avail = self.cols, self.ld, self.rd, self.avail
        t = avail * mone
        bit = t & avail
        pb = bit != 0
        avail = bit * mone + avail
        nc = bit * one + cols
        nl = bit * two + ld
        nr = sar1(rd | bit)
        na = ~(nc | nl | nr)
        pc = popc(nc)
        ps = pc > self.side_popc
        pl = pc == 31
        msk = np.where(pl, self.last_mask, self.noside)
        na = np.where(ps, na & msk, na)
        xl = nl * two
        xr = sar1(nr)
        f0 = ~(nc | xl | xr)
        t = f0 * mone
        lo = t & f0
        ma = lo * m4
        pos = bfind(f0) * mone + np.uint32(33)
        mb = shr_clamp(mone, pos)
        na = np.where(~pl, na & (ma | mb), na)
        pd = (na != 0) & pb
        pe = nc == mone
        w = np.where(bit == self.tie_bit, self.w_tie, self.w)
        self.cnt += np.where(pe, w, 0).astype(np.uint64)
        pp = (avail != 0) & pd
        pq0 = (avail == 0) & ~pd
        lanes = np.arange(self.n)
        idx = lanes[pp]
        self.stack[idx, self.sp[idx]] = np.stack([cols[idx], ld[idx], rd[idx], avail[idx]], axis=1)
        self.sp[idx] += 1
        self.deepest = np.maximum(self.deepest, self.sp)
        cols = np.where(pd, nc, cols)
        ld = np.where(pd, xl, ld)
        rd = np.where(pd, nr, rd)
        avail = np.where(pd, na, avail)
        pq = (self.sp != 0) & pq0
        idx = lanes[pq]
        self.sp[idx] -= 1
        top = self.stack[idx, self.sp[idx]]
        cols[idx], ld[idx], rd[idx], avail[idx] = top[:, 0], top[:, 1], top[:, 2], top[:, 3]
        self.cols, self.ld, self.rd, self.avail = cols, ld, rd, avail

    run = Lanes.run


@pytest.mark.parametrize("N,k", [(4, 2), (5, 2), (6, 2), (7, 3), (8, 3), (9, 3), (10, 4), (11, 4), (12, 5), (13, 5)])
def test_dihedral_step_weighted_counts(N, k):
    c, l, r, cls, classes = oracle.dihedral_expand(N, k)
    lanes = DihLanes(N, c, l, r, cls, classes)
    got = lanes.run()
    np.testing.assert_array_equal(got, oracle.dihedral_count_tasks(N, k, c, l, r, cls))
    assert int(got.sum()) == oracle.total(N, min(2, N - 2))
    # The dihedral launch reserves N-1-popc(cols) slots (rows N-2 and N-1 are stepped).
    assert (lanes.deepest <= np.maximum(1, N - 1 - popc(c).astype(np.int64))).all()


def saved_levels(lanes):
    """The entries a deadline dump writes: the current level (if it has untried columns) and every stacked level,
    with the left diagonal back in the reference's form (ld >> 1)."""
    out = []
    for i in range(lanes.n):
        if lanes.avail[i]:
            out.append((lanes.cols[i], lanes.ld[i] >> np.uint32(1), lanes.rd[i], lanes.avail[i]))
        for s in range(lanes.sp[i]):
            x, y, z, w = lanes.stack[i, s]
            out.append((x, y >> np.uint32(1), z, w))
    return np.array(out, np.uint32).reshape(-1, 4)


@pytest.mark.parametrize("dihedral", [False, True])
def test_saved_levels_pass_the_checkpoint_check(dihedral):
    # The resumable entries refuse a checkpoint entry unless its column mask carries the off-board columns and
    # its untried columns are free; every level the kernel can save mid-run passes.
    N, k = 12, 4
    if dihedral:
        c, l, r, cls, classes = oracle.dihedral_expand(N, k)
        lanes = DihLanes(N, c, l, r, cls, classes)
    else:
        c, l, r = oracle.expand(N, k)
        lanes = Lanes(N, c, l, r)
    last = np.uint32((1 << N) - 1)
    seen = 0
    for _ in range(6):
        for _ in range(40):
            lanes.step()
        e = saved_levels(lanes)
        seen += len(e)
        assert ((e[:, 0] & ~last) == ~last).all()
        assert not (e[:, 3] & (e[:, 0] | e[:, 1] | e[:, 2])).any()
    assert seen > 1000
