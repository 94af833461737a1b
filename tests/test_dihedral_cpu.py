"""Dihedral (8-fold) decomposition: the oracle against known totals, and the
library's host expander against the oracle's (no GPU needed).

The decomposition has no counterpart in the reference; its only contract is
the reference's whole-board total (README.md:16-25, logs/5090.log), which the
oracle's plain total is pinned to in test_oracle.py.
"""
import json
import os

import numpy as np
import pytest

import n_queens_b200 as nq
import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _known(N):
    pub = json.load(open(os.path.join(GOLDEN, "published.json")))
    if str(N) in pub:
        return pub[str(N)]["total"]
    return oracle.total(N, 2 if N >= 4 else 1)


@pytest.mark.parametrize("N", range(4, 15))
def test_oracle_dihedral_total_every_depth(N):
    want = _known(N)
    for k in range(2, N - 1):
        assert oracle.dihedral_total(N, k) == want, (N, k)


@pytest.mark.parametrize("N,k", [(15, 4), (15, 5), (16, 5), (16, 6), (17, 6)])
def test_oracle_dihedral_total_larger(N, k):
    assert oracle.dihedral_total(N, k) == _known(N)


@pytest.mark.parametrize("N,k", [(4, 2), (5, 3), (8, 3), (9, 4), (12, 5), (13, 6), (16, 5), (19, 6), (21, 6),
                                 (22, 7)])
def test_host_expander_matches_oracle(N, k):
    c, l, r, cls, classes = nq.dihedral_expand(N, k)
    oc, ol, orr, ocls, ocl = oracle.dihedral_expand(N, k)
    assert c.size == oc.size
    assert np.array_equal(c, oc) and np.array_equal(l, ol) and np.array_equal(r, orr)
    assert np.array_equal(cls, ocls)
    assert [(x["side_row"], x["last_mask"], x["tie_bit"], x["weight"], x["weight_tie"]) for x in classes] == ocl


def test_dihedral_task_counts():
    # 1.75x fewer DFS nodes needs no more tasks than the mirror decomposition
    # at the same depth by more than a small factor.
    for N, k in ((16, 5), (21, 6)):
        n_dih = nq.dihedral_expand(N, k)[0].size
        n_ref = nq.expand(N, k)[0].size
        assert 0.3 * n_ref < n_dih < 1.2 * n_ref, (N, k, n_dih, n_ref)


@pytest.mark.parametrize("N,k", [(3, 1), (4, 1), (4, 3), (8, 7), (32, 6), (10, 0)])
def test_dihedral_rejects_bad_arguments(N, k):
    with pytest.raises(nq.NQError):
        nq.dihedral_expand(N, k)
    with pytest.raises(nq.NQError):
        nq.count_dihedral(N, k)


def _solutions(N):
    out, q = [], []

    def rec(row, cols, d1, d2):
        if row == N:
            out.append(tuple(q))
            return
        for c in range(N):
            if c in cols or (row + c) in d1 or (row - c) in d2:
                continue
            q.append(c)
            rec(row + 1, cols | {c}, d1 | {row + c}, d2 | {row - c})
            q.pop()

    rec(0, frozenset(), frozenset(), frozenset())
    return out


def _images(q):
    N = len(q)
    cells = [(r, c) for r, c in enumerate(q)]
    maps = [lambda r, c: (r, c), lambda r, c: (c, N - 1 - r), lambda r, c: (N - 1 - r, N - 1 - c),
            lambda r, c: (N - 1 - c, r), lambda r, c: (r, N - 1 - c), lambda r, c: (N - 1 - r, c),
            lambda r, c: (c, r), lambda r, c: (N - 1 - c, N - 1 - r)]
    imgs = set()
    for f in maps:
        b = [0] * N
        for r, c in cells:
            rr, cc = f(r, c)
            b[rr] = cc
        imgs.add(tuple(b))
    return imgs


@pytest.mark.parametrize("N", range(6, 12))
def test_every_orbit_gets_its_size(N):
    # Each solution is counted by the tasks whose prefix it extends, under their
    # classes' rules and weights; over every orbit of the eight symmetries of the
    # square the weights must add up to the orbit's size.
    sols = _solutions(N)
    for k in range(2, min(6, N - 1)):
        c, l, r, cls, classes = oracle.dihedral_expand(N, k)
        by_prefix = {}
        for i in range(c.size):
            by_prefix.setdefault((int(c[i]), int(l[i]), int(r[i])), []).append(classes[int(cls[i])])
        weight = {}
        for q in sols:
            cc = ll = rr = 0
            for i in range(k):
                p = 1 << q[i]
                cc, ll, rr = cc | p, ((ll | p) << 1) & 0xFFFFFFFF, (rr | p) >> 1
            w = 0
            for side_row, last_mask, tie_bit, wt, wt_tie in by_prefix.get((cc, ll, rr), []):
                if any(i > side_row and q[i] in (0, N - 1) for i in range(k, N)):
                    continue
                last = 1 << q[N - 1]
                if not last & last_mask:
                    continue
                w += wt_tie if last == tie_bit else wt
            weight[q] = w
        seen = set()
        for q in sols:
            if q in seen:
                continue
            orbit = _images(q)
            seen |= orbit
            assert sum(weight[s] for s in orbit) == len(orbit), (N, k, q)


def test_resumable_checkpoint_mode_is_checked(tmp_path):
    # Read before any device work, so this runs without a GPU.
    import ctypes
    import struct
    p = tmp_path / "ck"
    t = ctypes.c_uint64(0)
    d = ctypes.c_int(0)

    def hdr(mode):
        return b"NQB200CK" + struct.pack("<IiiiqqQQq", 1, 10, 3, mode, 100, 5, 7, 1, 0)

    p.write_bytes(hdr(0))                                     # a plain count's checkpoint
    assert nq.lib.nq_count_dihedral_resumable(10, 3, None, str(p).encode(), ctypes.byref(t), ctypes.byref(d),
                                              None) == nq.NQ_ERR_ARG
    assert "plain" in nq.last_error()
    p.write_bytes(hdr(1))                                     # a dihedral count's checkpoint
    assert nq.lib.nq_count_resumable(10, 3, None, str(p).encode(), ctypes.byref(t), ctypes.byref(d),
                                     None) == nq.NQ_ERR_ARG
    assert "dihedral" in nq.last_error()
    p.write_bytes(hdr(2))                                     # unknown mode
    assert nq.lib.nq_count_dihedral_resumable(10, 3, None, str(p).encode(), ctypes.byref(t), ctypes.byref(d),
                                              None) == nq.NQ_ERR_ARG
    one = b"NQB200CK" + struct.pack("<IiiiqqQQq", 1, 10, 3, 1, 100, 5, 7, 1, 1) + bytes(16)
    p.write_bytes(one)                                        # an entry without its class byte
    assert nq.lib.nq_count_dihedral_resumable(10, 3, None, str(p).encode(), ctypes.byref(t), ctypes.byref(d),
                                              None) == nq.NQ_ERR_ARG


def test_resumable_checkpoint_entries_are_checked(tmp_path):
    # A continuation entry must carry the off-board columns and list only free columns as untried; anything
    # else is refused before any device work (a valid file gets as far as the missing device).
    import ctypes
    import struct
    p = tmp_path / "ck"
    t = ctypes.c_uint64(0)
    d = ctypes.c_int(0)
    N, rows = 10, 3
    off = 0xFFFFFFFF & ~((1 << N) - 1)
    ntasks = nq.expand(N, rows)[0].size

    def write(entries):
        hdr = b"NQB200CK" + struct.pack("<IiiiqqQQq", 1, N, rows, 0, ntasks, 5, 7, 1, len(entries))
        p.write_bytes(hdr + b"".join(struct.pack("<IIII", *e) for e in entries))

    def run():
        return nq.lib.nq_count_resumable(N, rows, None, str(p).encode(), ctypes.byref(t), ctypes.byref(d), None)

    good = (off | 0b1, 0b10, 0, 0b1100)          # a queen in column 0; columns 2 and 3 untried
    for bad in [(0b1, 0b10, 0, 0b1100),          # off-board columns missing
                (off | 0b1, 0b10, 0, 0b1101),    # untried column 0 is taken
                (off | 0b1, 0b110, 0, 0b1100),   # untried column 2 is on a left diagonal
                (off | 0b1, 0b10, 0b1000, 0b1100)]:  # untried column 3 is on a right diagonal
        write([good, bad])
        assert run() == nq.NQ_ERR_ARG, bad
        assert "continuation entry" in nq.last_error()
    write([good])
    assert run() in (nq.NQ_ERR_NO_DEVICE, nq.NQ_OK)
    # A header that promises more entries than the file holds is refused without sizing buffers for them.
    hdr = b"NQB200CK" + struct.pack("<IiiiqqQQq", 1, N, rows, 0, ntasks, 5, 7, 1, (1 << 32) - 1)
    p.write_bytes(hdr + struct.pack("<IIII", *good))
    assert run() == nq.NQ_ERR_ARG
    assert "not a valid checkpoint" in nq.last_error()
