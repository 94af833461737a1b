#!/usr/bin/env python
"""bench.py -- DFS nodes/s and wall ms of the B200 N-Queens counting path.

One step counts a whole board on one GPU: every half-board prefix of `k` rows
(the reference's task list, src/n_queens.cpp:74-113) goes through the
persistent DFS kernel, and the step's count is checked bit-exact against the
reference's published total (README.md / logs).  The default workload is
N=21, k=6 (4,470,757 prefix tasks).

Two queue orders are timed, interleaved step by step: the learned
longest-first order (the default headline: an MLP cost model built once per
run from solver-logged node counts, then a device-side predict + sort inside
every step) and the plain dynamic fetch in expander order (`compare`).

Reported (one JSON line from rank 0):
  value      DFS nodes/s with the tasks resident in HBM (schedule + queue
             reset + kernel, CUDA events on the launching stream, L2 flushed
             between steps);
  e2e        the same metric through the public API (learned:
             nq_count_learned; plain: nq_count): host expansion, pinned H2D
             copy of the tasks, schedule, kernel, D2H of the result; host wall
             clock per step;
  roofline   integer-issue roofline: 22 warp-issue slots per DFS node against
             numSMs x 4 schedulers x clock;
  cpu_baseline  the reference's own CPU recursion (oracle/_ref, all host
             threads) on a seeded sample of the same tasks.
  dihedral   the same whole-board count through the 8-fold decomposition
             (nq_count_dihedral, prefix depth k+1), timed through the public
             API after the measured arms; it visits fewer DFS nodes, so it is
             reported as time per count, not in `value`.

`--impl reference` times only that reference CPU path (rank 0; other ranks
exit 0).  Under torchrun each rank counts the same board on its own GPU
(replicas: the reference's multi-GPU split is out of scope), and the time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

I_ALG = 22  # algorithmic warp-issue slots per DFS node (fixed cost model)
METRIC = "DFS nodes/s (exact whole-board count, 1 B200)"

# Whole-board workloads: published totals (README.md:16-25, logs/5090.log) and
# DFS node totals (placements into rows k..N-2, counted by the node-counting
# kernel -- nq_count(..., nodes) -- and, up to N=17, by the CPU oracle).
WORKLOADS = {
    "n16k5": dict(N=16, k=5, total=14772512, nodes=563126914),
    "n17k6": dict(N=17, k=6, total=95815104, nodes=3959755915),
    "n18k6": dict(N=18, k=6, total=666090624, nodes=29348496950),
    "n19k6": dict(N=19, k=6, total=4968057848, nodes=228483606026),
    "n20k6": dict(N=20, k=6, total=39029188884, nodes=1865470950135),
    "n21k6": dict(N=21, k=6, total=314666222712, nodes=15916200586353),
    "n22k6": dict(N=22, k=6, total=2691008701644, nodes=141911885610183),
}


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="n21k6")
    ap.add_argument("--cpu-seconds", type=float, default=8.0, help="CPU work per reference-sample step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--schedule", choices=["learned", "plain"], default="learned",
                    help="queue order of the headline arm; the other order is timed beside it")
    ap.add_argument("--no-compare", action="store_true", help="skip timing the other queue order")
    ap.add_argument("--no-dihedral", action="store_true", help="skip timing the dihedral decomposition")
    ap.add_argument("--no-n22", action="store_true",
                    help="skip the N=22 k=6 learned-vs-plain pair (run after the N=21 default workload)")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU binary (oracle/_ref/n_queens_ref) on this GPU")
    ap.add_argument("--no-build-e2e", action="store_true",
                    help="skip the end-to-end learned count that includes building the cost model")
    return ap.parse_args()


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms while running (clocks and throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
            if self.gpu_id:
                cmd += ["-i", self.gpu_id]
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
                except ValueError:
                    continue
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        reasons = sorted({n for _, _, flags in rows for n, f in zip(self.NAMES, flags) if f.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- CPU reference sample
def reference_sample(N: int, k: int, seconds: float, seed: int = 12345):
    """A seeded random sample of the workload's prefix tasks sized for about
    `seconds` of the reference's CPU recursion on all host threads; returns
    (aos int32[n,3], nodes, counts, threads, kind)."""
    import oracle

    cols, ld, rd = oracle.expand(N, k)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(cols.size)
    threads = os.cpu_count() or 1
    kind = "reference" if oracle.ref_available() else "port"

    def run(idx):
        aos = np.stack([cols[idx], ld[idx], rd[idx]], axis=1).view(np.int32)
        t = time.perf_counter()
        if kind == "reference":
            oracle.ref_count_tasks(N, aos, threads=threads)
        else:
            oracle.count_tasks(N, cols[idx], ld[idx], rd[idx], threads=threads)
        return time.perf_counter() - t

    n = 4 * threads
    while True:
        dt = run(perm[:n])
        if dt > 0.5 or n >= cols.size:
            break
        n = min(cols.size, n * 4)
    n = int(min(cols.size, max(n, n * seconds / max(dt, 1e-3))))
    idx = np.sort(perm[:n])
    cnt, nodes = oracle.count_tasks(N, cols[idx], ld[idx], rd[idx], nodes=True, threads=threads)
    aos = np.stack([cols[idx], ld[idx], rd[idx]], axis=1).view(np.int32)
    return aos, int(nodes.sum()), cnt, threads, kind


def reference_sample_text(N, k, n, ntasks, nodes, threads, kind):
    how = ("the reference's own n_queens() recursion (src/n_queens.cpp:8-21, compiled unchanged into "
           "oracle/_ref/libnq_ref.so) called per task by the shim nqref_count_tasks with OpenMP "
           f"schedule(dynamic,1) on {threads} threads -- not parallel_n_queens's hard-coded 32 threads with "
           "static scheduling (src/n_queens.cpp:152-153)"
           if kind == "reference" else
           f"the C restatement of the reference recursion (oracle/nq_oracle.c) on {threads} threads")
    return (f"{n} of {ntasks} N={N} k={k} prefix tasks (seeded uniform sample, {nodes} DFS nodes) through "
            f"{how}, on {cpu_model()}")


def time_reference(N, aos, threads, kind, cnt):
    import oracle

    t = time.perf_counter()
    if kind == "reference":
        s2, per = oracle.ref_count_tasks(N, aos, threads=threads, per_task=True)
        ok = np.array_equal(per.view(np.uint64), cnt)
    else:
        c = aos.view(np.uint32)
        per = oracle.count_tasks(N, c[:, 0], c[:, 1], c[:, 2], threads=threads)
        ok = np.array_equal(per, cnt)
    dt = time.perf_counter() - t
    if not ok:
        raise SystemExit("reference sample: per-task counts disagree with the oracle")
    return dt


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ----------------------------------------------------------------------------- distributed
def dist_init(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist

        if n_gpus > 0:
            import torch

            torch.cuda.set_device(local)  # each rank's NCCL communicator on its own GPU
        dist.init_process_group("nccl" if n_gpus > 0 else "gloo", timeout=datetime.timedelta(seconds=900))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def traffic_from_profile(name: str):
    """DRAM bytes per launch of the DFS kernel, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ----------------------------------------------------------------------------- reference GPU binary
def parse_reference_log(text: str):
    """(start-job stamps, finish-job stamps, result, calc ms) from the
    reference CLI's output: "[YYYY-mm-dd HH:MM:SS.mmm] " lines
    (src/utils.cpp:14-30), "gpu [i] start job" / "gpu [i] finish job"
    (src/n_queens_cuda.cu:154,178) and the result line (src/main.cpp:53)."""
    import re

    stamp = re.compile(r"^\[(\d{4}-\d\d-\d\d \d\d:\d\d:\d\d\.\d{3})\] (.*)$")

    def when(t):
        return datetime.datetime.strptime(t, "%Y-%m-%d %H:%M:%S.%f").timestamp()

    starts, finishes, result, calc_ms = [], [], None, None
    for line in text.splitlines():
        m = stamp.match(line.strip())
        if not m:
            continue
        body = m.group(2)
        if "start job" in body:
            starts.append(when(m.group(1)))
        elif "finish job" in body:
            finishes.append(when(m.group(1)))
        rm = re.search(r"queens result (-?\d+), calc time: \[([0-9.]+)ms\]", body)
        if rm:
            result, calc_ms = int(rm.group(1)), float(rm.group(2))
    return starts, finishes, result, calc_ms


def reference_gpu_run(N: int, k: int, want: int, local: int) -> dict:
    """The reference's own CLI + CUDA kernel (oracle/_ref/n_queens_ref: its
    src/ files compiled unchanged for sm_100a, CONFIG2) on this rank's GPU,
    one count per process (its queue word, src/n_queens_cuda.cu:8, is never
    reset).  Job time = its "start job" to "finish job" log lines
    (src/n_queens_cuda.cu:154,178); calc time = its own result line
    (src/main.cpp:50-53), which also covers context creation and the host
    expansion."""
    exe = os.path.join(ROOT, "oracle", "_ref", "n_queens_ref")
    if not os.path.exists(exe):
        return {"ran": False, "why": "oracle/_ref/n_queens_ref was not built (needs the reference sources)"}
    env = dict(os.environ)
    vis = env.get("CUDA_VISIBLE_DEVICES")
    env["CUDA_VISIBLE_DEVICES"] = vis.split(",")[local] if vis else str(local)
    t0 = time.perf_counter()
    try:
        p = subprocess.run([exe, str(N), str(k)], capture_output=True, text=True, env=env, timeout=900)
    except subprocess.TimeoutExpired:
        return {"ran": False, "why": "timed out after 900 s"}
    wall = time.perf_counter() - t0
    starts, finishes, result, calc_ms = parse_reference_log(p.stdout)
    out = {"ran": True, "rc": p.returncode, "binary": "oracle/_ref/n_queens_ref (CONFIG2: 160 threads x 19 levels)",
           "N": N, "k": k, "count": result, "count_ok": result == want, "calc_ms": calc_ms,
           "process_wall_ms": 1000 * wall, "gpus_used": len(starts)}
    if starts and finishes:
        out["job_ms"] = 1000 * (max(finishes) - min(starts))
    if result != want:
        out["stdout_tail"] = p.stdout[-400:]
    return out


# ----------------------------------------------------------------------------- arms
def run_reference(args, world, rank):
    wl = WORKLOADS[args.workload]
    if rank != 0:
        return
    N, k = wl["N"], wl["k"]
    aos, nodes, cnt, threads, kind = reference_sample(N, k, args.cpu_seconds)
    for _ in range(args.warmup):
        time_reference(N, aos, threads, kind, cnt)
    times = [time_reference(N, aos, threads, kind, cnt) for _ in range(args.steps)]
    total = sum(times)
    value = nodes * args.steps / total
    sample = reference_sample_text(N, k, aos.shape[0], oracle_tasks(N, k), nodes, threads, kind)
    line = {
        "metric": METRIC, "value": value, "unit": "nodes/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 masks / u64 counts",
        "data": "synthetic (the reference's own prefix tasks; deterministic)",
        "config": {"workload": f"N={N} k={k} whole-board count", "N": N, "k": k, "tasks_per_step": int(aos.shape[0])},
        "cpu_baseline": {"value": value, "unit": "nodes/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "nodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def oracle_tasks(N, k):
    import oracle

    return int(oracle.lib.nq_oracle_expand(N, k, None, None, None, 0))


def run_ours(args, world, rank, local):
    import torch

    import n_queens_b200 as nq

    wl = WORKLOADS[args.workload]
    N, k, want = wl["N"], wl["k"], wl["total"]
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    props = torch.cuda.get_device_properties(dev)
    sms = props.multi_processor_count
    gpu_uuid = None
    try:
        gpu_uuid = "GPU-" + str(props.uuid)
    except Exception:
        pass

    # Tasks resident in HBM for the device-timed loop.
    cols, ld, rd = nq.expand(N, k)
    ntasks = cols.size
    tc = torch.from_numpy(cols.view(np.int32)).to(dev)
    tl = torch.from_numpy(ld.view(np.int32)).to(dev)
    tr = torch.from_numpy(rd.view(np.int32)).to(dev)
    levels = nq.stack_levels(N, k)  # stack slots per lane of the count kernel for k-row prefixes
    cfg = nq.Config()
    cfg.device = local
    cfg.stack_levels = levels
    stream = torch.cuda.current_stream(dev)
    nslots = max(args.steps, args.warmup, 1)
    sums = torch.zeros((nslots, 2), dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    nodes = wl["nodes"]
    if nodes is None:
        r = nq.count(N, k, config=cfg, nodes=True)
        assert r.total == want, (r.total, want)
        nodes = r.nodes

    # Learned longest-first order: the cost model is built once (solver-logged
    # labels at N=16..18, fine-tuning on a seeded 5% sample of this board);
    # every learned step then predicts + sorts on the device and counts.
    model, build = None, None
    order = torch.empty(ntasks, dtype=torch.int32, device=dev)
    lcfg = nq.Config()
    lcfg.device = local
    lcfg.stack_levels = levels
    lcfg.order_kind = nq.NQ_ORDER_GIVEN
    lcfg.order = order.data_ptr()
    want_learned = args.schedule == "learned" or not args.no_compare
    if want_learned:
        from n_queens_b200 import learned
        t0 = time.perf_counter()
        model, rep = learned.build_cost_model(N, k=k, seed=1, device=local)
        build = {"wall_s": time.perf_counter() - t0, "label_s": rep.label_s, "pretrain_s": rep.pretrain_s,
                 "finetune_label_s": rep.finetune_label_s, "finetune_s": rep.finetune_s,
                 "train_samples": rep.train_samples, "finetune_samples": rep.finetune_samples,
                 "holdout_spearman": rep.holdout_spearman, "holdout_rmse_log2": rep.holdout_rmse}

    def check(nsteps):
        s = sums[:nsteps].cpu().numpy()
        for i in range(nsteps):
            if 2 * int(s[i, 0]) != want or int(s[i, 1]) != 0:
                raise SystemExit(f"step {i}: count {2 * int(s[i, 0])} status {int(s[i, 1])}, want {want}")

    def step(i, kind, mid=None):
        sp = sums[i]
        c = cfg
        if kind == "learned":
            rc = learned.lib.nq_schedule_device(model._m, N, tc.data_ptr(), tl.data_ptr(), tr.data_ptr(), ntasks,
                                                order.data_ptr(), None, stream.cuda_stream)
            if rc != 0:
                raise SystemExit(f"nq_schedule_device: {nq.status_string(rc)} {nq.last_error()}")
            c = lcfg
        if mid is not None:
            mid.record(stream)
        rc = nq.lib.nq_count_tasks_device(N, tc.data_ptr(), tl.data_ptr(), tr.data_ptr(), ntasks, None, None,
                                          sp.data_ptr(), nq.ctypes.byref(c), stream.cuda_stream)
        if rc != 0:
            raise SystemExit(f"nq_count_tasks_device: {nq.status_string(rc)} {nq.last_error()}")

    head = args.schedule
    other = None if args.no_compare else ("plain" if head == "learned" else "learned")
    for i in range(args.warmup):
        flush.zero_()
        step(i, head)
    torch.cuda.synchronize()
    check(args.warmup)

    # Timed: the headline order and (interleaved, same conditions) the other.
    arms = [head] + ([other] if other else [])
    ev = {a: [tuple(torch.cuda.Event(enable_timing=True) for _ in range(3)) for _ in range(args.steps)]
          for a in arms}
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(gpu_uuid) as clk:
        for i in range(args.steps):
            for a in arms:
                flush.zero_()
                ev[a][i][0].record(stream)
                step(i, a, mid=ev[a][i][1])
                ev[a][i][2].record(stream)
            torch.cuda.synchronize()
            check(i + 1)
    barrier(world)
    clocks = clk.summary()
    arm_s = {a: sum(s.elapsed_time(e) for s, _, e in ev[a]) / 1000.0 for a in arms}
    dfs_s = sum(m.elapsed_time(e) for _, m, e in ev[head]) / 1000.0  # the DFS kernel alone
    sched_ms = (arm_s[head] - dfs_s) * 1000.0 / args.steps
    t_local = arm_s[head]
    t_max = max_over_ranks(world, t_local)
    value = world * nodes * args.steps / t_max
    compare = None
    if other:
        o_max = max_over_ranks(world, arm_s[other])
        compare = {"schedule": other, "value": world * nodes * args.steps / o_max,
                   "ms_per_step": 1000 * o_max / args.steps,
                   "headline_speedup": o_max / t_max}

    # End to end through the public C ABI (nq_count_learned / nq_count):
    # expansion, pinned H2D, schedule, kernel, D2H of the result words and of
    # the per-CTA start/end stamps (nq_config.timing: makespan and tail idle).
    def e2e_arm(kind, nsteps):
        ecfg = nq.Config()
        ecfg.device = local
        ecfg.timing = 1

        def one():
            if kind == "learned":
                return learned.count_learned(N, k, model, config=ecfg)
            return nq.count(N, k, config=ecfg)

        r = one()  # sizes the library's buffers for this board
        if r.total != want:
            raise SystemExit(f"e2e {kind}: count {r.total}, want {want}")
        barrier(world)
        walls, stats = [], []
        for i in range(nsteps):
            t0 = time.perf_counter()
            r = one()
            walls.append(time.perf_counter() - t0)
            if r.total != want:
                raise SystemExit(f"e2e {kind} step {i}: count {r.total}, want {want}")
            stats.append(r.stats)
        barrier(world)
        e_max = max_over_ranks(world, sum(walls))
        grid = int(stats[-1]["grid"])
        return {
            "value": world * nodes * nsteps / e_max, "unit": "nodes/s", "steps": nsteps,
            "wall_ms_per_step": 1000 * e_max / nsteps,
            "h2d_bytes_per_step": 12 * ntasks, "d2h_bytes_per_step": 24 + 16 * grid,
            "breakdown_ms": {key: statistics.mean(s[key] for s in stats)
                             for key in ("expand_ms", "h2d_ms", "schedule_ms", "kernel_ms", "d2h_ms", "total_ms")},
            "tail_idle_frac": statistics.mean(s["tail_idle_frac"] for s in stats),
            "makespan_ms": statistics.mean(s["makespan_ms"] for s in stats),
            "grid": grid, "block_threads": int(stats[-1]["block_threads"]),
            "api": "n_queens_b200.learned.count_learned (nq_count_learned)" if kind == "learned"
                   else "n_queens_b200.count (nq_count)",
        }

    e2e = e2e_other = None
    if not args.no_e2e:
        e2e = e2e_arm(head, args.steps)
        if other:
            e2e_other = e2e_arm(other, min(args.steps, 3))
            e2e_other["schedule"] = other
    if compare is not None and e2e is not None:
        compare.update({
            "makespan_ms": {head: e2e["makespan_ms"], other: e2e_other["makespan_ms"]},
            "tail_idle_frac": {head: e2e["tail_idle_frac"], other: e2e_other["tail_idle_frac"]},
            "e2e_wall_ms_per_step": {head: e2e["wall_ms_per_step"], other: e2e_other["wall_ms_per_step"]},
            "note": "makespan and tail idle: per-CTA %globaltimer stamps of the e2e counts (nq_config.timing)"})

    # The learned path with its model built inside the timed region: build
    # (labels at N=16..18, pre-training, a labelled 5% fine-tuning sample and
    # hold-out of this board), then the count of the tasks the build did not
    # already count (nq_count_learned_reuse), against the plain e2e count.
    build_e2e = None
    if want_learned and not args.no_e2e and not args.no_build_e2e:
        barrier(world)
        t0 = time.perf_counter()
        m2, rep2 = learned.build_cost_model(N, k=k, seed=2, device=local)
        t_build = time.perf_counter() - t0
        bcfg = nq.Config()
        bcfg.device = local
        bcfg.timing = 1
        r = learned.count_learned(N, k, m2, config=bcfg, reuse=rep2)
        wall = time.perf_counter() - t0
        m2.close()
        if r.total != want:
            raise SystemExit(f"learned count with the model build: {r.total}, want {want}")
        wall = max_over_ranks(world, wall)
        plain_ms = e2e_other["wall_ms_per_step"] if (e2e_other and other == "plain") else (
            e2e["wall_ms_per_step"] if head == "plain" else None)
        build_e2e = {"wall_ms": 1000 * wall, "model_build_ms": 1000 * t_build,
                     "count_wall_ms": 1000 * wall - 1000 * t_build, "kernel_ms": r.stats["kernel_ms"],
                     "tasks_counted_by_build": int(rep2.counted_idx.size), "queue_tasks": int(ntasks - rep2.counted_idx.size),
                     "count_ok": True, "plain_e2e_wall_ms": plain_ms,
                     "speedup_vs_plain_e2e": (plain_ms / (1000 * wall)) if plain_ms else None,
                     "api": "n_queens_b200.learned.build_cost_model + count_learned(reuse=...) "
                            "(nq_count_learned_reuse)"}

    # The same count through the 8-fold decomposition (fewer nodes, same
    # total): wall and kernel time per count through nq_count_dihedral.
    dihedral = None
    if not args.no_dihedral and N >= 6:
        kd = min(k + 1, N - 2)
        dcfg = nq.Config()
        dcfg.device = local
        r = nq.count_dihedral(N, kd, config=dcfg)  # sizes the buffers
        if r.total != want:
            raise SystemExit(f"dihedral: count {r.total}, want {want}")
        barrier(world)
        walls, kms = [], []
        dsteps = min(args.steps, 3)
        for i in range(dsteps):
            t0 = time.perf_counter()
            r = nq.count_dihedral(N, kd, config=dcfg)
            walls.append(time.perf_counter() - t0)
            if r.total != want:
                raise SystemExit(f"dihedral step {i}: count {r.total}, want {want}")
            kms.append(r.stats["kernel_ms"])
        barrier(world)
        d_max = max_over_ranks(world, sum(walls))
        dihedral = {"rows": kd, "tasks": int(r.stats["tasks"]), "count_ok": True, "steps": dsteps,
                    "wall_ms_per_step": 1000 * d_max / dsteps, "kernel_ms_per_step": statistics.mean(kms),
                    "speedup_vs_headline_step": (1000 * t_max / args.steps) / (1000 * d_max / dsteps),
                    "api": "n_queens_b200.count_dihedral (nq_count_dihedral)"}

    # The configuration the large-board target is quoted on: N=22, k=6,
    # learned (model built once for N=22) then plain, each checked against the
    # published total, with makespan and tail idle.
    n22 = None
    if args.workload == "n21k6" and not args.no_n22 and want_learned:
        w22 = WORKLOADS["n22k6"]
        barrier(world)
        t0 = time.perf_counter()
        m22, _ = learned.build_cost_model(22, k=6, seed=1, device=local)
        b22 = time.perf_counter() - t0
        runs = {}
        for kind in ("learned", "plain"):
            c22 = nq.Config()
            c22.device = local
            c22.timing = 1
            barrier(world)
            t0 = time.perf_counter()
            r = learned.count_learned(22, 6, m22, config=c22) if kind == "learned" else nq.count(22, 6, config=c22)
            wall = max_over_ranks(world, time.perf_counter() - t0)
            if r.total != w22["total"]:
                raise SystemExit(f"N=22 {kind}: count {r.total}, want {w22['total']}")
            st = r.stats
            runs[kind] = {"count": int(r.total), "count_ok": True, "tasks": int(st["tasks"]), "wall_ms": 1000 * wall,
                          "kernel_ms": st["kernel_ms"], "schedule_ms": st["schedule_ms"],
                          "makespan_ms": st["makespan_ms"], "tail_idle_frac": st["tail_idle_frac"],
                          "block_threads": int(st["block_threads"]), "grid": int(st["grid"])}
            if w22["nodes"]:
                runs[kind]["nodes_per_s_kernel"] = w22["nodes"] / (st["kernel_ms"] / 1000.0)
                runs[kind]["nodes_per_s_wall"] = world * w22["nodes"] / wall
        m22.close()
        n22 = {"N": 22, "k": 6, "tasks": runs["plain"]["tasks"], "count": w22["total"],
               "dfs_nodes": w22["nodes"], "model_build_ms": 1000 * b22,
               "learned": runs["learned"], "plain": runs["plain"],
               "kernel_speedup_learned_over_plain": runs["plain"]["kernel_ms"] / runs["learned"]["kernel_ms"],
               "wall_speedup_learned_over_plain": runs["plain"]["wall_ms"] / runs["learned"]["wall_ms"],
               "api": "count_learned (nq_count_learned) then count (nq_count), nq_config.timing = 1"}

    ref_gpu = None
    if world == 1 and not args.no_reference_gpu:
        ref_gpu = reference_gpu_run(N, k, want, local)
        if ref_gpu.get("job_ms"):
            ref_gpu["headline_step_speedup_vs_job"] = ref_gpu["job_ms"] / (1000 * t_max / args.steps)

    peak_clock = None
    try:
        peak_clock = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("sm_max_mhz")
    except (OSError, ValueError):
        pass
    peak_src = "MEASURED_PEAKS.json sm_max_mhz"
    if not peak_clock:
        peak_clock, peak_src = clocks.get("sm_max_mhz") or 1965.0, "sampled clocks.max.sm"
    achieved = (nodes * args.steps / dfs_s) * I_ALG / 32 / 1e9
    peak = sms * 4 * peak_clock * 1e6 / 1e9
    roof = {
        "bound": "int-issue", "achieved": achieved, "peak": peak, "unit": "Gwarp-inst/s", "frac": achieved / peak,
        "traffic": traffic_from_profile(f"dfs_kernel_n{N}k{k}.md"),
        "kernel_ms_per_launch": 1000 * dfs_s / args.steps,
        "note": (f"achieved = DFS nodes/s of the DFS kernel alone x {I_ALG} issue slots / 32 lanes; "
                 f"peak = {sms} SMs x 4 schedulers x "
                 f"{peak_clock:.0f} MHz ({peak_src}); traffic = ncu DRAM bytes per launch"),
    }
    if clocks.get("sm_mhz"):
        roof["frac_at_sampled_clock"] = achieved / (sms * 4 * clocks["sm_mhz"] * 1e6 / 1e9)
    if n22 is not None:
        for arm in ("learned", "plain"):
            r22 = n22[arm]
            if "nodes_per_s_kernel" in r22:
                r22["roofline_frac"] = r22["nodes_per_s_kernel"] * I_ALG / 32 / 1e9 / peak

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        aos, snodes, cnt, threads, kind = reference_sample(N, k, args.cpu_seconds)
        dt = time_reference(N, aos, threads, kind, cnt)
        cpu = {"value": snodes / dt, "unit": "nodes/s", "cores": threads, "kind": kind,
               "sample": reference_sample_text(N, k, aos.shape[0], ntasks, snodes, threads, kind)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "nodes/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 masks / u64 counts",
            "data": "synthetic (the reference's own prefix tasks; deterministic)",
            "config": {"workload": f"N={N} k={k} whole-board count", "N": N, "k": k, "tasks": int(ntasks),
                       "dfs_nodes": int(nodes), "count": int(want),
                       "schedule": ("learned longest-first (MLP cost model, device predict + sort inside each step)"
                                    if head == "learned" else "plain dynamic fetch"),
                       "l2": "flushed (256 MiB write) between timed steps", "parallelism": f"replicas x{world}",
                       "stack_levels": levels},
            "e2e": e2e, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
            "compare": compare, "e2e_other": e2e_other, "build_e2e": build_e2e, "dihedral": dihedral,
            "n22": n22, "reference_gpu": ref_gpu, "model_build": build, "schedule_ms_per_step": sched_ms,
            # our kernels per timed step: learned = predict + bin + DFS (the radix sort between
            # them is CUB's), plain = DFS
            "gpu_launches": sum(args.steps * (3 if a == "learned" else 1) for a in arms),
        }
        print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    world, rank, local = dist_init(args.gpus if args.impl == "ours" else 0)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
