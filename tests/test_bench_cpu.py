"""bench.py's host logic on CPU: the reference arm (the reference's own CPU
recursion, no GPU needed), alone and under torchrun with two gloo ranks, and
the max-over-ranks timing reduction."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["--impl", "reference", "--workload", "n16k5", "--steps", "1", "--warmup", "1", "--cpu-seconds", "0.3"]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _json_lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def test_reference_arm_line():
    r = subprocess.run([sys.executable, "bench.py", *ARGS], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "nodes/s"
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["config"]["N"] == 16 and d["steps"] == 1 and d["warmup"] == 1


def test_reference_arm_loads_no_product_library():
    # The reference arm must run only the reference's code (oracle/_ref) and
    # the checkers; the product library may not even be mapped.
    code = ("import runpy, sys; sys.argv = ['bench.py'] + %r; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('PRODUCT_MAPPED' if 'libnqueens_b200' in maps else 'PRODUCT_NOT_MAPPED')" % (ARGS,))
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "PRODUCT_NOT_MAPPED" in r.stdout
    d = _json_lines(r.stdout)[0]
    if d["cpu_baseline"]["kind"] == "reference":
        assert "schedule(dynamic,1)" in d["cpu_baseline"]["sample"]


def test_reference_log_parser():
    # The reference CLI's timestamped lines (src/utils.cpp:14-30), its job
    # lines (src/n_queens_cuda.cu:154,178) and result line (src/main.cpp:53).
    sys.path.insert(0, ROOT)
    import bench
    text = ("[2026-01-02 03:04:05.000] ====\n"
            "[2026-01-02 03:04:05.080] Use 80.00ms to generate 4470757 subproblems!\n"
            "[2026-01-02 03:04:06.250] gpu [0] start job, with 4470757(1.000) subproblems.\n"
            "[2026-01-02 03:04:32.050] gpu [0] finish job.\n"
            "[2026-01-02 03:04:32.100] cuda 21 queens result 314666222712, calc time: [27100.00ms]\n")
    starts, finishes, result, calc = bench.parse_reference_log(text)
    assert result == 314666222712 and calc == 27100.0
    assert len(starts) == 1 and len(finishes) == 1
    assert abs((finishes[0] - starts[0]) - 25.8) < 1e-6


def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--gpus", "2", *ARGS]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1 and lines[0]["impl"] == "reference"   # rank 0 alone prints


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, _ = bench.dist_init(0)
    bench.barrier(w)
    q.put((r, bench.max_over_ranks(w, 1.5 + r)))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 2.5, 1: 2.5}


def test_reference_cpu_solver_timing_script():
    # oracle.time_reference_cpu times the reference's own parallel_n_queens
    # (oracle/_ref); where the reference was not built it says so and exits.
    sys.path.insert(0, ROOT)
    import oracle
    r = subprocess.run([sys.executable, "-m", "oracle.time_reference_cpu", "--N", "12", "--k", "4"], cwd=ROOT,
                       capture_output=True, text=True, timeout=300)
    if not oracle.ref_available():
        assert r.returncode != 0 and "not built" in (r.stderr + r.stdout)
        return
    assert r.returncode == 0, r.stderr
    d = _json_lines(r.stdout)[0]
    assert d["solver"] == "parallel_n_queens" and d["total"] == 14200 and d["total_ok"]
    assert d["omp_threads"] == 32 and d["host_cores"] >= 1 and d["seconds"] >= 0
