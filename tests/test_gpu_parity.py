"""GPU parity: every count through the C ABI, bit-exact against the oracle
(oracle/, pinned to the reference) or the reference's published totals."""
import numpy as np
import pytest

import oracle
from n_queens_b200 import workloads

pytestmark = pytest.mark.gpu


def test_whole_board_small_n_all_k(gpu):
    for N in range(4, 15):
        for k in range(1, N - 1):
            r = gpu.count(N, k)
            assert r.total == oracle.total(N, k), (N, k)


def test_odd_n_one_row_keeps_reference_value(gpu, golden):
    # For odd N and rows == 1 the reference's expander emits the middle-column
    # board without the second-row restriction, so its x2 sum overcounts
    # (serial_n_queens(5, 1) == 12, not 10).  The CLI never gets there (it
    # raises rows to 2, src/main.cpp:26-29); the library returns the
    # reference's value for the same (N, rows).
    ref = {(c["N"], c["k"]): c["total"] for c in golden("totals_ref.json")}
    for N in (5, 7, 9, 11):
        assert gpu.count(N, 1).total == ref[(N, 1)]
        assert gpu.count(N, 2).total == oracle.total(N, 2)


def test_whole_board_published(gpu, golden):
    pub = golden("published.json")
    for N, k in [(13, 5), (14, 5), (15, 5), (16, 5), (16, 6), (17, 6), (18, 6), (19, 6)]:
        assert gpu.count(N, k).total == pub[str(N)]["total"], (N, k)
        assert gpu.cuda_n_queens(N, k) == pub[str(N)]["total"]


def test_nodes_match_oracle(gpu):
    table = {(12, 4): 418_515, (16, 5): 563_126_914, (16, 6): 562_707_506, (17, 6): 3_959_755_915}
    for (N, k), nodes in table.items():
        r = gpu.count(N, k, nodes=True)
        assert r.nodes == nodes, (N, k)
    for N, k in [(9, 3), (10, 4), (11, 3), (13, 5)]:
        want_total, want_nodes = oracle.total(N, k, with_nodes=True)
        r = gpu.count(N, k, nodes=True)
        assert (r.total, r.nodes) == (want_total, want_nodes), (N, k)


def test_per_task_counts_and_nodes(gpu):
    for N, k in [(10, 3), (12, 4), (13, 5), (15, 5)]:
        c, l, r = oracle.expand(N, k)
        want_cnt, want_nodes = oracle.count_tasks(N, c, l, r, nodes=True)
        res = gpu.count_tasks(N, c, l, r, per_task=True, nodes=True)
        assert np.array_equal(res["per_task"], want_cnt), (N, k)
        assert np.array_equal(res["nodes"], want_nodes), (N, k)
        assert res["sum"] == int(want_cnt.sum())


def test_per_task_golden_hashes(gpu, golden):
    import hashlib
    for case in golden("per_task.json"):
        c, l, r = oracle.expand(case["N"], case["k"])
        res = gpu.count_tasks(case["N"], c, l, r, per_task=True)
        got = res["per_task"].astype(np.int64)
        assert hashlib.sha256(got.tobytes()).hexdigest() == case["sha256_counts_int64"], case
        assert 2 * res["sum"] == case["sum_x2"]


def test_arbitrary_32bit_inputs(gpu):
    # Whatever bits the caller passes, the count is the reference recursion's.
    rng = np.random.default_rng(11)
    for N in (1, 2, 5, 8, 10, 12):
        n = 4000
        cols = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        cols &= rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        cols &= rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        keep = rng.random(n) < 0.7
        cols[keep] &= np.uint32((1 << N) - 1)
        ld = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32) & rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        rd = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32) & rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        want = oracle.count_tasks(N, cols, ld, rd)
        res = gpu.count_tasks(N, cols, ld, rd, per_task=True)
        assert np.array_equal(res["per_task"], want), N


def test_arbitrary_inputs_on_large_boards(gpu):
    # Boards up to N=31 with one to nine columns left, arbitrary diagonal bits
    # (a right mask with bit 31 set shifts arithmetically, as the reference's
    # int does) and some column masks with off-board bits: the count step's
    # filter works on the top bit positions here (bits 29-31 of its masks).
    rng = np.random.default_rng(29)
    for N in (20, 24, 28, 30, 31):
        n = 3000
        last = (1 << N) - 1
        cols = np.empty(n, np.uint32)
        for i in range(n):
            left = int(rng.integers(1, 10))
            free = rng.choice(N, left, replace=False)
            cols[i] = last & ~int(sum(1 << int(f) for f in free))
        off = rng.random(n) < 0.1
        cols[off] |= np.uint32(1 << (31 if N == 31 else N + int(rng.integers(0, 32 - N))))
        r32 = lambda: rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        ld = r32() & r32()
        rd = r32() & r32()
        rd[rng.random(n) < 0.3] |= np.uint32(0x80000000)
        want = oracle.count_tasks(N, cols, ld, rd)
        res = gpu.count_tasks(N, cols, ld, rd, per_task=True)
        assert np.array_equal(res["per_task"], want), N


def test_edge_tasks(gpu):
    N = 8
    last = (1 << N) - 1
    cols = np.array([last, last | 256, 0, 0b1, 0xFF00, 0], np.uint32)
    ld = np.array([0, 0, 0, 0, 0, 0xFF], np.uint32)
    rd = np.array([0, 0, 0, 0, 0, 0], np.uint32)
    want = oracle.count_tasks(N, cols, ld, rd)
    assert list(want) == [1, 0, 92, oracle.count_task(8, 1, 0, 0), 0, 0]
    res = gpu.count_tasks(N, cols, ld, rd, per_task=True)
    assert np.array_equal(res["per_task"], want)
    empty = gpu.count_tasks(N, [], [], [], per_task=True)
    assert empty["sum"] == 0 and empty["per_task"].size == 0


def test_launch_shapes_and_order_give_same_count(gpu, golden):
    pub = golden("published.json")
    N, k = 17, 6
    c, l, r = oracle.expand(N, k)
    want = pub[str(N)]["total"]
    for cfg in [dict(block_threads=64), dict(block_threads=128, blocks_per_sm=1), dict(block_threads=512),
                dict(steal=-1), dict(inner_steps=4), dict(inner_steps=1024), dict(stack_levels=20)]:
        assert 2 * gpu.count_tasks(N, c, l, r, config=cfg)["sum"] == want, cfg
    perm = np.random.default_rng(2).permutation(c.size).astype(np.uint32)
    cfg = gpu.Config()
    cfg.order_kind = gpu.NQ_ORDER_GIVEN
    cfg.order = perm.ctypes.data
    res = gpu.count_tasks(N, c, l, r, per_task=True, config=cfg)
    assert 2 * res["sum"] == want
    assert np.array_equal(res["per_task"], oracle.count_tasks(N, c, l, r))


def test_depth_error_is_reported(gpu):
    with pytest.raises(gpu.NQError) as e:
        gpu.count(16, 5, config=dict(stack_levels=3))
    assert e.value.status == gpu.NQ_ERR_DEPTH
    # The context stays usable.
    assert gpu.count(12, 4).total == 14200


def test_config_upper_bounds(gpu):
    for bad in (dict(inner_steps=gpu.NQ_MAX_INNER_STEPS + 1), dict(stack_levels=gpu.NQ_MAX_STACK_LEVELS + 1),
                dict(stack_levels=1 << 18, block_threads=1024)):
        with pytest.raises(gpu.NQError) as e:
            gpu.count(12, 4, config=bad)
        assert e.value.status == gpu.NQ_ERR_ARG, bad
    # The bounds themselves are accepted, and the context stays usable.
    assert gpu.count(12, 4, config=dict(inner_steps=gpu.NQ_MAX_INNER_STEPS)).total == 14200
    assert gpu.count(12, 4, config=dict(stack_levels=gpu.NQ_MAX_STACK_LEVELS)).total == 14200


def test_time_limit_stops_kernel_and_context_survives(gpu, golden):
    with pytest.raises(gpu.NQError) as e:
        gpu.count(19, 6, config=dict(time_limit_ms=1))
    assert e.value.status == gpu.NQ_ERR_TIMEOUT
    assert gpu.count(13, 5).total == golden("published.json")["13"]["total"]


def test_device_entry_with_torch_tensors(gpu, golden):
    import torch
    N, k = 16, 5
    c, l, r = oracle.expand(N, k)
    dev = torch.device("cuda:0")
    tc = torch.from_numpy(c.view(np.int32)).to(dev)
    tl = torch.from_numpy(l.view(np.int32)).to(dev)
    tr = torch.from_numpy(r.view(np.int32)).to(dev)
    out = torch.zeros(2, dtype=torch.int64, device=dev)
    per = torch.zeros(c.size, dtype=torch.int64, device=dev)
    gpu.count_tasks_device(N, tc, tl, tr, out, per_task=per, config=dict(stack_levels=N - 1 - k),
                           stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    assert 2 * int(out[0]) == golden("published.json")[str(N)]["total"]
    assert int(out[1]) == 0
    assert np.array_equal(per.cpu().numpy().view(np.uint64), oracle.count_tasks(N, c, l, r))
    # Too few stack levels: the status word says so.
    gpu.count_tasks_device(N, tc, tl, tr, out, config=dict(stack_levels=2), stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    assert int(out[1]) & 1


def test_batch_small_boards(gpu, golden):
    g = golden("boards_small.json")
    inst = [tuple(b) for b in g["instances"]]
    for split in (0, 1, 3, 5):
        out = gpu.count_batch(inst, split_rows=split)
        assert out.tolist() == g["counts"], split


def test_dropin_n_queens_single_board(gpu):
    for (N, c, l, r) in workloads.random_boards(20, 9, 8, 15, 0, 4):
        assert gpu.n_queens(N, c, l, r) == oracle.count_task(N, c, l, r)


def test_cli_result_line(gpu):
    import subprocess
    out = subprocess.run([gpu.CLI_PATH, "16", "5"], capture_output=True, text=True, timeout=300).stdout
    assert "cuda 16 queens result 14772512, calc time: [" in out
    assert "to generate 70906 subproblems!" in out
    assert "gpu [0] start job, with 70906(1.00) subproblems." in out


def test_batch_dedup_and_symmetry(gpu):
    # Duplicates, mirror images, empty boards (symmetric: half-board rule)
    # and a symmetric odd board with a middle queen, all against the oracle.
    boards = []
    for N in range(4, 13):
        boards.append((N, 0, 0, 0))
        if N % 2:
            p = 1 << (N // 2)
            boards.append((N, p, p << 1, p >> 1))
    base = workloads.random_boards(120, 21, 8, 13, 0, 5)
    boards += base + base[:30]
    boards += [(N,) + workloads.mirror_board(N, c, l, r) for (N, c, l, r) in base[30:60]]
    want = [oracle.count_task(*b) for b in boards]
    for cfg in (None, dict(layout=1), dict(block_threads=64)):
        for split in (0, 1, 4, 7):
            assert gpu.count_batch(boards, split_rows=split, config=cfg).tolist() == want, (cfg, split)


def test_batch_plan_replays(gpu, golden):
    g = golden("boards_small.json")
    inst = [tuple(b) for b in g["instances"]]
    plan = gpu.BatchPlan(inst, split_rows=4)
    for _ in range(3):
        out, st = plan.run(return_stats=True)
        assert out.tolist() == g["counts"]
        assert st["tasks"] > 0 and st["kernel_ms"] > 0
    plan.close()


def test_batch_autotune_sweep(gpu):
    inst = workloads.random_boards(96, 4, 9, 13, 0, 3)
    want = [oracle.count_task(*b) for b in inst]
    best, table = gpu.autotune_batch(inst, repeats=1)
    assert len(table) == 42
    assert {e["split_rows"] for e in table} == {3, 4, 5, 6, 7}
    assert {e["block_threads"] for e in table} == {64, 128, 256, 512}
    assert {e["layout"] for e in table} == {0, 1}
    assert {e["inner_steps"] for e in table} == {256, 1024, 4096}
    # the chunking stage runs at the fastest entry of the first stage
    first = min(table[:40], key=lambda e: e["ms"])
    assert all((e["split_rows"], e["block_threads"], e["layout"]) ==
               (first["split_rows"], first["block_threads"], first["layout"]) for e in table[40:])
    assert best["ms"] == min(e["ms"] for e in table)
    cfg = dict(block_threads=best["block_threads"], layout=best["layout"], inner_steps=best["inner_steps"])
    assert gpu.count_batch(inst, split_rows=best["split_rows"], config=cfg).tolist() == want


def test_device_expander_matches_reference_bytes(gpu, golden):
    import ctypes
    import hashlib
    import torch
    dev = torch.device("cuda:0")
    for case in golden("expander.json"):
        N, k = case["N"], case["k"]
        n = ctypes.c_int64(0)
        assert gpu.lib.nq_expand_device(N, k, None, None, None, 0, ctypes.byref(n), 0, None) == 0
        assert n.value == case["tasks"], case
        bufs = [torch.empty(max(n.value, 1), dtype=torch.int32, device=dev) for _ in range(3)]
        assert gpu.lib.nq_expand_device(N, k, *(b.data_ptr() for b in bufs), n.value, ctypes.byref(n), 0,
                                        None) == 0
        torch.cuda.synchronize()
        aos = np.stack([b[:n.value].cpu().numpy() for b in bufs], axis=1)
        assert hashlib.sha256(np.ascontiguousarray(aos).tobytes()).hexdigest() == case["sha256_aos_int32"], case


def test_count_with_device_expansion(gpu, golden):
    pub = golden("published.json")
    for N, k in [(13, 5), (16, 6), (19, 6)]:
        r = gpu.count(N, k, config=dict(device_expand=1))
        assert r.total == pub[str(N)]["total"] and r.stats["tasks"] > 0
    for N in range(4, 12):
        for k in range(1, N - 1):
            assert gpu.count(N, k, config=dict(device_expand=1)).total == oracle.total(N, k), (N, k)
