"""Measures the batched workload: 4096 uneven partial boards in one
graph-captured persistent launch (N uniform in [12, 20], 0-4 random queens in
the top rows, seed 1 -- n_queens_b200.workloads.random_boards).

    python -m n_queens_b200.batch_bench [--tune-boards 512] [--repeats 3] [--json out.json]

1. autotunes split depth / CTA size / stack layout / queue chunking (nq_batch_autotune) on a
   cheaper batch of the same shape (N in [12, 17], seed 2);
2. builds the 4096-board plan with the winner and times graph replays;
3. prints the plan's statistics and a checksum of the 4096 counts.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import time

import numpy as np

from . import BatchPlan, autotune_batch
from .workloads import random_boards


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tune-boards", type=int, default=512)
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--json", default=None)
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
    print(json.dumps({k: v for k, v in res.items() if k != "autotune_table"}), flush=True)
    if args.json:
        with open(args.json, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
