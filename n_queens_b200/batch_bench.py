"""Measures the batched workload: 4096 uneven partial boards in one
graph-captured persistent launch (N uniform in [12, 20], 0-4 random queens in
the top rows, seed 1 -- n_queens_b200.workloads.random_boards).

    python -m n_queens_b200.batch_bench [--tune-boards 512] [--repeats 3] [--json out.json] [--nodes]

1. autotunes split depth / CTA size / stack layout / queue chunking (nq_batch_autotune) on a
   cheaper batch of the same shape (N in [12, 17], seed 2);
2. builds the 4096-board plan with the winner and times graph replays;
3. prints the plan's statistics and a checksum of the 4096 counts;
4. with --nodes, estimates the DFS nodes one replay visits (plan_nodes) and
   reports the replay's node rate against the integer-issue roofline.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import time

import numpy as np

from . import BatchPlan, autotune_batch, count_tasks
from .workloads import mirror_board, random_boards

I_ALG = 22  # warp-issue slots per DFS node (the roofline's cost model)


def plan_nodes(boards, split_rows: int) -> float:
    """Estimated DFS nodes of a batch plan's subtasks.

    Mirrors the plan: distinct boards up to mirror image, each split
    `split_rows` rows deeper; the subtasks' nodes are counted on the GPU
    (nq_count_tasks with per-task nodes) and a mirror-symmetric board, whose
    plan keeps only its left half, counts half of its nodes (exact for even N;
    for odd N the middle column is halved again one row down, which this
    treats as exact).
    """
    canon = {}
    for (N, c, l, r) in boards:
        key = (N, c, l, r)
        mk = (N,) + tuple(mirror_board(N, c, l, r))
        canon[min(key, mk)] = mk == key
    by_n = {}
    for (N, c, l, r), sym in canon.items():
        by_n.setdefault(N, []).append((c, l, r, sym))
    total = 0.0
    for N, lst in sorted(by_n.items()):
        last = np.uint64((1 << N) - 1)
        c = np.array([x[0] for x in lst], np.uint64)
        l = np.array([x[1] for x in lst], np.uint64)
        r = np.array([x[2] for x in lst], np.uint64)
        owner = np.arange(len(lst))
        for _ in range(split_rows):
            free = ~(c | l | r) & last
            done = c == last
            parts = [(c[done], l[done], r[done], owner[done])]
            for b in range(N):
                p = np.uint64(1 << b)
                sel = ((free >> np.uint64(b)) & np.uint64(1)).astype(bool) & ~done
                parts.append((c[sel] | p, ((l[sel] | p) << np.uint64(1)) & np.uint64(0xFFFFFFFF),
                              (r[sel] | p) >> np.uint64(1), owner[sel]))
            c, l, r, owner = (np.concatenate([q[i] for q in parts]) for i in range(4))
        res = count_tasks(N, c.astype(np.uint32), l.astype(np.uint32), r.astype(np.uint32), nodes=True)
        per_board = np.bincount(owner, weights=res["nodes"].astype(np.float64), minlength=len(lst))
        total += float((per_board * np.array([0.5 if x[3] else 1.0 for x in lst])).sum())
    return total


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tune-boards", type=int, default=512)
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--json", default=None)
    ap.add_argument("--nodes", action="store_true", help="estimate the replay's DFS nodes and node rate")
    args = ap.parse_args()
    tune = random_boards(args.tune_boards, 2, 12, 17, 0, 4)
    t = time.perf_counter()
    best, table = autotune_batch(tune, repeats=2)
    tune_s = time.perf_counter() - t
    print(json.dumps({"autotune_s": tune_s, "best": best}), flush=True)
    boards = random_boards(4096, 1, 12, 20, 0, 4)
    t = time.perf_counter()
    plan = BatchPlan(boards, split_rows=best["split_rows"],
                     config=dict(block_threads=best["block_threads"], layout=best["layout"],
                                 inner_steps=best["inner_steps"]))
    build_s = time.perf_counter() - t
    runs = []
    out = None
    for _ in range(args.repeats + 1):
        t = time.perf_counter()
        out, st = plan.run(return_stats=True)
        runs.append(dict(wall_s=time.perf_counter() - t, kernel_ms=st["kernel_ms"], tasks=st["tasks"],
                         grid=st["grid"], block_threads=st["block_threads"], stack_levels=st["stack_levels"]))
    plan.close()
    res = {"boards": len(boards), "plan_build_s": build_s, "warmup": runs[0], "timed": runs[1:],
           "kernel_ms_mean": float(np.mean([r["kernel_ms"] for r in runs[1:]])),
           "counts_sum": int(out.sum()), "counts_sha256": hashlib.sha256(out.tobytes()).hexdigest(),
           "autotune_best": best, "autotune_table": table, "autotune_s": tune_s}
    if args.nodes:
        import torch
        props = torch.cuda.get_device_properties(0)
        try:
            mhz = json.load(open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                              "MEASURED_PEAKS.json")))["sm_max_mhz"]
        except (OSError, ValueError, KeyError):
            mhz = props.clock_rate / 1000.0
        nodes = plan_nodes(boards, best["split_rows"])
        rate = nodes / (res["kernel_ms_mean"] / 1e3)
        res.update(dfs_nodes_est=nodes, nodes_per_s=rate,
                   int_issue_frac=rate * I_ALG / 32 / (props.multi_processor_count * 4 * mhz * 1e6))
    print(json.dumps({k: v for k, v in res.items() if k != "autotune_table"}), flush=True)
    if args.json:
        with open(args.json, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
