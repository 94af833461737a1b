"""Whole-board count with the learned longest-first order against the plain
expander order, on one GPU (the comparison the cost model exists for).

    python -m n_queens_b200.compare_schedules --N 22 --k 6 [--repeats 1] [--json out.json]
                                              [--schedules plain,learned,dihedral]
                                              [--block-threads 0,192,512] [--reuse]

Builds the cost model once (solver-logged node counts at N=16..18, fine-tuned
on a seeded 5% sample of the target's prefixes), then alternates plain and
learned whole-board counts through the public API (nq_count and
nq_count_learned), each with per-CTA timing, and prints wall time, kernel
time, makespan, tail-idle fraction and the count of every run.  `dihedral`
adds the 8-fold decomposition (nq_count_dihedral) to the same alternation;
`--block-threads` alternates CTA sizes inside each schedule; `--reuse` makes
the learned counts skip the tasks that the model build already counted.
"""
from __future__ import annotations

import argparse
import json
import time

from . import count, count_dihedral
from . import learned


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=22)
    ap.add_argument("--k", type=int, default=6)
    ap.add_argument("--repeats", type=int, default=1)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--json", default=None)
    ap.add_argument("--schedules", default="plain,learned", help="comma list of plain, learned, dihedral")
    ap.add_argument("--block-threads", default="0",
                    help="comma list of CTA sizes to alternate (0 = the library's default choice)")
    ap.add_argument("--reuse", action="store_true",
                    help="learned counts skip the tasks the model build counted exactly (nq_count_learned_reuse)")
    args = ap.parse_args()
    threads = [int(x) for x in args.block_threads.split(",") if x]
    names = [x for x in args.schedules.split(",") if x]
    out = {"N": args.N, "k": args.k, "runs": []}
    model = rep = None
    if "learned" in names:
        t = time.perf_counter()
        model, rep = learned.build_cost_model(args.N, k=args.k, seed=args.seed)
        out.update(model_build_s=time.perf_counter() - t,
                   build={k: v for k, v in rep.__dict__.items() if k != "counted_idx"})
        print(json.dumps({"model_build_s": out["model_build_s"], "holdout_spearman": rep.holdout_spearman}),
              flush=True)
    for it in range(args.repeats):
        for name in names:
            for bt in threads:
                cfg = dict(timing=1, block_threads=bt)
                t = time.perf_counter()
                if name == "plain":
                    r = count(args.N, args.k, config=cfg)
                elif name == "dihedral":
                    r = count_dihedral(args.N, args.k, config=cfg)
                else:
                    r = learned.count_learned(args.N, args.k, model, config=cfg, reuse=rep if args.reuse else None)
                wall = time.perf_counter() - t
                st = r.stats
                row = {"schedule": name, "repeat": it, "total": r.total, "wall_s": wall,
                       "kernel_ms": st["kernel_ms"], "schedule_ms": st["schedule_ms"],
                       "makespan_ms": st["makespan_ms"], "tail_idle_frac": st["tail_idle_frac"],
                       "expand_ms": st["expand_ms"], "tasks": st["tasks"], "block_threads": st["block_threads"],
                       "grid": st["grid"], "stack_levels": st["stack_levels"]}
                out["runs"].append(row)
                print(json.dumps(row), flush=True)
    if args.json:
        with open(args.json, "w") as f:
            json.dump(out, f, indent=1)
    if model is not None:
        model.close()


if __name__ == "__main__":
    main()
