"""Pins the CPU oracle (oracle/nq_oracle.c) to the reference.

The golden fixtures were produced by the reference's own code compiled from
its sources (tests/golden/make_golden.py); published totals and task counts
come from the reference's README and logs.  When oracle/_ref is built here the
oracle is also compared with the reference live on random inputs.
"""
import hashlib

import numpy as np
import pytest

import oracle
from n_queens_b200 import workloads


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_expander_matches_reference_bytes(golden):
    for case in golden("expander.json"):
        if case["tasks"] > 3_000_000:
            continue
        c, l, r = oracle.expand(case["N"], case["k"])
        aos = np.stack([c, l, r], axis=1).view(np.int32)
        assert aos.shape[0] == case["tasks"], case
        assert sha(aos) == case["sha256_aos_int32"], case


def test_expander_task_counts_match_logs(golden):
    for case in golden("published_tasks.json")["cases"]:
        if case["tasks"] > 20_000_000:
            continue
        assert oracle.lib.nq_oracle_expand(case["N"], case["k"], None, None, None, 0) == case["tasks"], case


def test_totals_match_reference_serial(golden):
    for case in golden("totals_ref.json"):
        assert oracle.total(case["N"], case["k"]) == case["total"], case


def test_totals_match_published(golden):
    pub = golden("published.json")
    for N, k in [(13, 5), (14, 5), (15, 5), (16, 5), (16, 6)]:
        assert oracle.total(N, k) == pub[str(N)]["total"]


def test_per_task_counts_match_reference(golden):
    for case in golden("per_task.json"):
        if case["tasks"] > 200_000:
            continue
        c, l, r = oracle.expand(case["N"], case["k"])
        cnt = oracle.count_tasks(case["N"], c, l, r)
        assert int(cnt.sum()) * 2 == case["sum_x2"]
        assert sha(cnt.astype(np.int64)) == case["sha256_counts_int64"], case


def test_node_counts_match_probe_table():
    # DFS node totals of the reference kernel loop (src/n_queens_cuda.cu:39-72),
    # as tabulated by an independent probe: (N, k) -> nodes.
    table = {(12, 4): 418_515, (16, 5): 563_126_914, (16, 6): 562_707_506}
    for (N, k), nodes in table.items():
        assert oracle.total(N, k, with_nodes=True)[1] == nodes


def test_small_boards_match_reference(golden):
    g = golden("boards_small.json")
    assert [list(b) for b in workloads.random_boards(g["n"], g["seed"], *g["N_range"], *g["m_range"])] == \
        g["instances"]
    for (N, c, l, r), want in zip(g["instances"], g["counts"]):
        assert oracle.count_task(N, c, l, r) == want


def test_mirror_board_has_same_count():
    for (N, c, l, r) in workloads.random_boards(64, 3, 6, 12, 0, 5):
        assert oracle.count_task(N, c, l, r) == oracle.count_task(N, *workloads.mirror_board(N, c, l, r))


def test_complete_and_malformed_boards():
    # cur == last counts 1 (src/n_queens.cpp:10-13); off-board column bits can
    # never reach `last`, so they count 0.
    assert oracle.count_task(5, 0b11111, 0, 0) == 1
    assert oracle.count_task(5, 0b111111, 0, 0) == 0
    assert oracle.count_task(1, 0, 0, 0) == 1
    assert oracle.nodes_task(8, 0b11111111, 0, 0) == 0


@pytest.mark.skipif(not oracle.ref_available(), reason="reference sources were not available to build oracle/_ref")
def test_oracle_equals_reference_on_random_inputs():
    rng = np.random.default_rng(5)
    L = oracle.ref()
    for _ in range(3000):
        N = int(rng.integers(1, 11))
        cur, left, right = (int(x) for x in rng.integers(0, 2**32, 3, dtype=np.uint64))
        # Thin out the masks so that boards have free columns.
        cur &= int(rng.integers(0, 2**32, dtype=np.uint64)) & int(rng.integers(0, 2**32, dtype=np.uint64))
        if rng.random() < 0.5:
            cur &= (1 << N) - 1
        want = L.nqref_n_queens(N, np.int32(np.uint32(cur)).item(), np.int32(np.uint32(left)).item(),
                                np.int32(np.uint32(right)).item())
        assert oracle.count_task(N, cur, left, right) == want, (N, cur, left, right)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference sources were not available to build oracle/_ref")
def test_oracle_expander_equals_reference_live():
    for N in range(2, 15):
        for k in range(1, N - 1):
            c, l, r = oracle.expand(N, k)
            ref = oracle.ref_expand_aos(N, k)
            assert np.array_equal(np.stack([c, l, r], axis=1).view(np.int32), ref), (N, k)


def test_batch_fixture_against_oracle_and_published(golden):
    # The 4096-board fixture (reference n_queens() on every distinct board):
    # its instances replay from the seed, cheap boards agree with the oracle,
    # empty boards carry the published totals, and where every one-queen
    # board of an N is present their counts add up to the published total
    # (the row-0 decomposition).
    g = golden("boards_4096.json")
    pub = golden("published.json")
    assert [list(b) for b in workloads.random_boards(g["n"], g["seed"], *g["N_range"], *g["m_range"])] == \
        g["instances"]
    one_queen = {}
    cheap = []
    for (N, c, l, r), want in zip(g["instances"], g["counts"]):
        m = bin(c).count("1")
        if m == 0 and str(N) in pub:
            assert want == pub[str(N)]["total"]
        if m == 1:
            one_queen.setdefault(N, {})[c] = want
        if N <= 13 or (N <= 15 and m >= 2):
            cheap.append((N, c, l, r, want))
    for N, c, l, r, want in cheap:
        assert oracle.count_task(N, c, l, r) == want
    full = [N for N, d in one_queen.items() if len(d) == N]
    assert 20 in full
    for N in full:
        if str(N) in pub:
            assert sum(one_queen[N].values()) == pub[str(N)]["total"], N
