"""Generates the golden fixtures in this directory from the reference itself.

Every value here comes from the reference's own code, compiled unchanged from
its sources into ``oracle/_ref/libnq_ref.so`` (``make -C oracle REF_SRC=<reference>/src``): its
expander ``partial_n_queens`` / ``partial_n_queens_for_odd``
(src/n_queens.cpp:74-113), its recursion ``n_queens`` (src/n_queens.cpp:8-21)
and its ``serial_n_queens`` (src/n_queens.cpp:115-137).  The published totals
(``published.json``) are copied from the reference's README and run logs with
their line citations.

Usage (in a checkout where the reference sources were available to make)::

    python tests/golden/make_golden.py            # expander, totals, per-task
    python tests/golden/make_golden.py --boards   # + the batched-board counts (long: ~30 min on 8 cores)
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from n_queens_b200 import workloads  # noqa: E402

EXPANDER_CASES = [(2, 1), (4, 1), (4, 2), (5, 1), (5, 2), (5, 3), (6, 2), (6, 4), (7, 3), (7, 5), (8, 1), (8, 2),
                  (8, 6), (9, 2), (9, 3), (9, 7), (10, 4), (11, 4), (11, 5), (12, 4), (13, 5), (14, 5), (15, 5),
                  (16, 5), (16, 6), (17, 6), (18, 6), (19, 6), (20, 6), (21, 6)]
TOTAL_CASES = [(5, 1), (7, 1), (9, 1), (11, 1), (4, 2), (5, 2), (5, 3), (6, 2), (6, 4), (7, 3), (8, 2), (8, 3),
               (8, 6), (9, 3), (9, 7), (10, 4), (11, 4), (12, 4), (12, 5), (13, 5), (14, 5), (15, 5), (16, 5)]
PER_TASK_CASES = [(8, 2), (9, 3), (10, 4), (11, 5), (12, 4), (13, 5), (14, 4), (15, 5), (16, 5), (17, 6)]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def gen_expander():
    out = []
    for N, k in EXPANDER_CASES:
        aos = oracle.ref_expand_aos(N, k)
        out.append({"N": N, "k": k, "tasks": int(aos.shape[0]), "sha256_aos_int32": sha(aos),
                    "head": aos[:4].tolist(), "tail": aos[-2:].tolist()})
    return out


def gen_totals():
    L = oracle.ref()
    return [{"N": N, "k": k, "total": int(L.nqref_serial(N, k))} for N, k in TOTAL_CASES]


def gen_per_task():
    out = []
    for N, k in PER_TASK_CASES:
        aos = oracle.ref_expand_aos(N, k)
        s2, per = oracle.ref_count_tasks(N, aos, per_task=True)
        rec = {"N": N, "k": k, "tasks": int(aos.shape[0]), "sum_x2": s2, "sha256_counts_int64": sha(per)}
        if aos.shape[0] <= 64:
            rec["counts"] = per.tolist()
        out.append(rec)
    return out


def children(N: int, board, depth: int):
    """The boards n_queens() recurses into `depth` rows below `board`.

    One recursion step of src/n_queens.cpp:14-19: every free column p of the
    next row gives (cur|p, (left|p)<<1, (right|p)>>1).  n_queens() of a board
    is the sum of n_queens() over these children unless the board is already
    complete, so splitting here only spreads the reference's own recursion
    over more OpenMP iterations.
    """
    last = (1 << N) - 1
    out = [board]
    for _ in range(depth):
        nxt = []
        for (c, l, r) in out:
            if c == last:
                nxt.append((c, l, r))
                continue
            v = last & ~(c | l | r)
            while v:
                p = v & -v
                v ^= p
                nxt.append((c | p, ((l | p) << 1) & 0xFFFFFFFF, (r | p) >> 1))
        out = nxt
    return out


def gen_boards(n: int, seed: int, n_lo: int, n_hi: int, m_lo: int, m_hi: int, threads: int = 0):
    """Reference counts of a seeded batch of partial boards.

    Identical boards are counted once, and a board and its mirror image
    (workloads.mirror_board, same count) share one count.  Empty boards of
    N >= 17 take their totals from the reference's README (their recursion
    would take hours).  All other boards run through the reference's
    n_queens(); boards with N >= 17 and few queens are first split into
    their recursion children (see children()) so the OpenMP loop balances.
    """
    published = {int(k): v["total"] for k, v in json.load(open(os.path.join(HERE, "published.json"))).items()}
    boards = workloads.random_boards(n, seed, n_lo, n_hi, m_lo, m_hi)
    canon = {}
    for (N, c, l, r) in boards:
        key = (N, c, l, r)
        mk = (N,) + workloads.mirror_board(N, c, l, r)
        canon[key] = min(key, mk)
    todo = sorted(set(canon.values()), key=lambda b: (b[0], bin(b[1]).count("1")))
    counts = {}
    big = []
    for b in todo:
        N, c, l, r = b
        if c == 0 and l == 0 and r == 0 and N >= 17:
            counts[b] = published[N]
        else:
            big.append(b)
    # Group by N so each ctypes call is one OpenMP loop over many boards.
    byN = {}
    for b in big:
        byN.setdefault(b[0], []).append(b)
    for N in sorted(byN):
        lst = byN[N]
        pieces, owner = [], []
        for i, b in enumerate(lst):
            m = bin(b[1]).count("1")
            depth = max(0, min(3, N - 16 - m)) if N >= 17 else 0
            for ch in children(N, b[1:], depth):
                pieces.append(ch)
                owner.append(i)
        aos = np.array(pieces, dtype=np.uint32).reshape(-1, 3).view(np.int32)
        t = time.time()
        _, per = oracle.ref_count_tasks(N, aos, threads=threads, per_task=True)
        sums = np.zeros(len(lst), np.int64)
        np.add.at(sums, np.array(owner), per)
        print(f"  N={N}: {len(lst)} distinct boards ({len(pieces)} pieces) in {time.time() - t:.1f}s", flush=True)
        for b, v in zip(lst, sums.tolist()):
            counts[b] = int(v)
    return {"seed": seed, "n": n, "N_range": [n_lo, n_hi], "m_range": [m_lo, m_hi],
            "instances": [[b[0], b[1], b[2], b[3]] for b in boards],
            "counts": [counts[canon[b]] for b in boards]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--boards", action="store_true", help="also the 4096-board batch (long)")
    ap.add_argument("--threads", type=int, default=0)
    args = ap.parse_args()
    if not oracle.ref_available():
        sys.exit("oracle/_ref/libnq_ref.so is not built: run make -C oracle REF_SRC=<reference>/src")
    t = time.time()
    json.dump(gen_expander(), open(os.path.join(HERE, "expander.json"), "w"), indent=1)
    json.dump(gen_totals(), open(os.path.join(HERE, "totals_ref.json"), "w"), indent=1)
    json.dump(gen_per_task(), open(os.path.join(HERE, "per_task.json"), "w"), indent=1)
    small = gen_boards(256, 7, 6, 14, 0, 6, args.threads)
    json.dump(small, open(os.path.join(HERE, "boards_small.json"), "w"))
    print(f"fixtures written in {time.time() - t:.1f}s")
    if args.boards:
        big = gen_boards(4096, 1, 12, 20, 0, 4, args.threads)
        json.dump(big, open(os.path.join(HERE, "boards_4096.json"), "w"))
        print(f"4096-board fixture written in {time.time() - t:.1f}s")


if __name__ == "__main__":
    main()
