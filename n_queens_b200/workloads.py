"""Seeded synthetic workloads for the counting path.

The reference publishes no dataset: its workloads are whole boards (N, k).
The batched workload of uneven partial boards is defined here so that tests,
golden fixtures and bench.py draw exactly the same instances.

Random partial boards (``random_boards``): for each instance draw N uniformly
from [n_lo, n_hi] and m uniformly from [m_lo, m_hi], then place m queens in
rows 0..m-1, each in a column drawn uniformly among the row's free columns;
if a row has no free column the instance is redrawn from row 0.  Each board is
packed as the reference packs a prefix (``src/n_queens.cpp:84-86``):
``(cur|p, (left|p)<<1, (right|p)>>1)``.  Its count is ``n_queens(N, cur,
left, right)`` of ``src/n_queens.cpp:8-21`` -- no symmetry factor.

The generator is SplitMix64 (Steele, Lea & Flood, "Fast splittable
pseudorandom number generators", OOPSLA 2014), so any language can replay it.
"""
from __future__ import annotations

import numpy as np

_M64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.state = seed & _M64

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _M64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
        return z ^ (z >> 31)

    def below(self, n: int) -> int:
        """Uniform integer in [0, n) (modulo draw; n is tiny so the bias is < 2^-58)."""
        return self.next() % n


def _nth_bit(mask: int, k: int) -> int:
    """The k-th (0-based) set bit of mask, as a one-bit mask."""
    for _ in range(k):
        mask &= mask - 1
    return mask & -mask


def random_board(rng: SplitMix64, N: int, m: int):
    """m random non-attacking queens in rows 0..m-1 of an N board, packed as a task."""
    last = (1 << N) - 1
    while True:
        cur = left = right = 0
        ok = True
        for _ in range(m):
            free = last & ~(cur | left | right)
            if free == 0:
                ok = False
                break
            p = _nth_bit(free, rng.below(bin(free).count("1")))
            cur |= p
            left = ((left | p) << 1) & 0xFFFFFFFF
            right = (right | p) >> 1
        if ok:
            return cur, left, right


def random_boards(n: int, seed: int = 1, n_lo: int = 12, n_hi: int = 20, m_lo: int = 0, m_hi: int = 4):
    """``n`` instances as a list of (N, cols, ld, rd)."""
    rng = SplitMix64(seed)
    out = []
    for _ in range(n):
        N = n_lo + rng.below(n_hi - n_lo + 1)
        m = m_lo + rng.below(m_hi - m_lo + 1)
        c, l, r = random_board(rng, N, m)
        out.append((N, c, l, r))
    return out


def boards_array(boards) -> np.ndarray:
    """(N, cols, ld, rd) tuples as a uint32[n, 4] array."""
    return np.array([[b[0], b[1], b[2], b[3]] for b in boards], dtype=np.uint32).reshape(-1, 4)


def mirror_board(N: int, cols: int, ld: int, rd: int):
    """Left-right mirror image of a packed board (same completion count).

    Column j maps to N-1-j; the left and right diagonal attack sets swap and
    reflect.  Bits of ld at or above N (attacks that already left the board)
    have no mirror counterpart and are dropped, which does not change the
    count because they can never return to the board.
    """
    def rev(x: int) -> int:
        y = 0
        for j in range(N):
            if x >> j & 1:
                y |= 1 << (N - 1 - j)
        return y

    last = (1 << N) - 1
    return rev(cols & last), rev(rd & last), rev(ld & last)
