"""CPU-side tests of the product library: symbols, host expander, argument
checks, the no-GPU behaviour of the drop-in entries and the CLI messages."""
import ctypes
import hashlib
import os
import re
import subprocess

import numpy as np
import pytest

import n_queens_b200 as nq
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def header_symbols():
    text = open(os.path.join(ROOT, "include", "n_queens_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(nq_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    syms = header_symbols()
    assert len(syms) >= 9
    for s in syms:
        assert hasattr(nq.lib, s), s
    assert set(nq.EXPORTS) == set(syms)
    assert nq.lib.nq_abi_version() == 1


def test_header_constants_match_python_mirror():
    text = open(os.path.join(ROOT, "include", "n_queens_b200.h")).read()
    defines = dict(re.findall(r"^#define (NQ_\w+) (.+)$", text, re.M))
    assert int(defines["NQ_MAX_N"]) == nq.NQ_MAX_N
    assert eval(defines["NQ_MAX_INNER_STEPS"]) == nq.NQ_MAX_INNER_STEPS
    assert int(defines["NQ_MAX_STACK_LEVELS"]) == nq.NQ_MAX_STACK_LEVELS
    # No task of a board of at most NQ_MAX_N columns needs more slots than the bound.
    assert max(nq.stack_levels(N, 0, nodes) for N in range(1, nq.NQ_MAX_N + 1) for nodes in (0, 1)) \
        <= nq.NQ_MAX_STACK_LEVELS
    assert int(defines["NQ_ABI_VERSION"]) == 1


def test_dropin_cxx_symbols_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", nq.LIB_PATH], capture_output=True, text=True).stdout
    for mangled in ["_Z13cuda_n_queensii", "_Z8n_queensiiiiRx"]:
        assert mangled in out, mangled
    assert "partial_n_queens" in out and "partial_n_queens_for_odd" in out


def test_host_expander_matches_reference_bytes(golden):
    for case in golden("expander.json"):
        for threads in (1, 0):
            c, l, r = nq.expand(case["N"], case["k"], threads=threads)
            aos = np.stack([c, l, r], axis=1).view(np.int32)
            assert aos.shape[0] == case["tasks"]
            assert sha(aos) == case["sha256_aos_int32"], (case["N"], case["k"], threads)


def test_host_expander_equals_oracle_for_every_small_case():
    # Every (N, k) up to N=20, k=6 and three thread counts: the parallel expander keeps the reference's order.
    for N in range(2, 21):
        for k in range(1, min(N, 6) + 1):
            want = oracle.expand(N, k)
            for threads in (1, 3, 0):
                got = nq.expand(N, k, threads=threads)
                for g, w in zip(got, want):
                    assert np.array_equal(g, w), (N, k, threads)


def test_host_expander_task_counts_match_logs(golden):
    for case in golden("published_tasks.json")["cases"]:
        n = ctypes.c_int64(0)
        assert nq.lib.nq_expand(case["N"], case["k"], None, None, None, 0, ctypes.byref(n), 0) == 0
        assert n.value == case["tasks"], case


def test_expand_partial_capacity():
    c, l, r = nq.expand(12, 4)
    cap = 100
    cc = np.zeros(cap, np.uint32)
    ll = np.zeros(cap, np.uint32)
    rr = np.zeros(cap, np.uint32)
    n = ctypes.c_int64(0)
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    assert nq.lib.nq_expand(12, 4, p(cc), p(ll), p(rr), cap, ctypes.byref(n), 3) == 0
    assert n.value == c.size
    assert np.array_equal(cc, c[:cap]) and np.array_equal(ll, l[:cap]) and np.array_equal(rr, r[:cap])


@pytest.mark.parametrize("N,k", [(1, 1), (32, 4), (8, 0), (8, 9), (-3, 2)])
def test_expand_rejects_bad_arguments(N, k):
    n = ctypes.c_int64(0)
    assert nq.lib.nq_expand(N, k, None, None, None, 0, ctypes.byref(n), 0) == nq.NQ_ERR_ARG


@pytest.mark.parametrize("N,k", [(1, 1), (8, 7), (8, 0), (32, 5)])
def test_count_rejects_bad_arguments(N, k):
    t = ctypes.c_uint64(0)
    assert nq.lib.nq_count(N, k, None, ctypes.byref(t), None, None) == nq.NQ_ERR_ARG


def test_count_rejects_null_output():
    assert nq.lib.nq_count(8, 2, None, None, None, None) == nq.NQ_ERR_ARG
    assert nq.lib.nq_count_tasks(8, None, None, None, 0, None, None, None, None, None) == nq.NQ_ERR_ARG


def test_status_strings():
    for s in range(-7, 1):
        assert nq.status_string(s) and nq.status_string(s) != "unknown status"
    assert nq.status_string(-99) == "unknown status"


def _no_gpu():
    try:
        return nq.device_count() == 0
    except nq.NQError:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="checks the no-GPU path")
def test_no_gpu_behaviour_matches_reference():
    # cuda_n_queens returns -1 when no GPU is found (src/n_queens_cuda.cu:105-108),
    # after generating the prefixes.
    assert nq.cuda_n_queens(12, 4) == -1
    st = nq.Stats()
    t = ctypes.c_uint64(0)
    assert nq.lib.nq_count(12, 4, None, ctypes.byref(t), None, ctypes.byref(st)) == nq.NQ_ERR_NO_DEVICE
    assert st.tasks == 2040
    with pytest.raises(nq.NQError) as e:
        nq.count_tasks(8, [0], [0], [0])
    assert e.value.status == nq.NQ_ERR_NO_DEVICE


def run_cli(*args):
    return subprocess.run([nq.CLI_PATH, *map(str, args)], capture_output=True, text=True, timeout=120)


def test_cli_argument_messages():
    # Messages of src/main.cpp:10-29.
    assert "Not allowed 1 queens problem!" in run_cli(1, 2).stdout
    assert "Not allowed 29 queens problem!" in run_cli(29, 6).stdout
    assert "Pre-placed rows should be <= 6." in run_cli(8, 7).stdout
    r = run_cli(8, 1)
    assert "Pre-placed rows shold be at least 2, so set to 2!" in r.stdout


@pytest.mark.skipif(not _no_gpu(), reason="checks the no-GPU path")
def test_cli_without_gpu():
    out = run_cli(12, 4).stdout
    assert "Use " in out and "to generate 2040 subproblems!" in out
    assert "Failed to find any gpu!" in out
    assert re.search(r"^\[\d{4}-\d\d-\d\d \d\d:\d\d:\d\d\.\d{3}\] cuda 12 queens result -1, calc time: \[",
                     out, re.M)


@pytest.mark.skipif(not _no_gpu(), reason="checks the no-GPU path")
def test_cli_dihedral_without_gpu(tmp_path):
    ck = tmp_path / "d.ckpt"
    for extra in ([], ["--checkpoint", str(ck), "--slice-ms", "5"]):
        out = run_cli(12, 4, "--dihedral", *extra).stdout
        assert "n_queens_b200: no CUDA device" in out
        assert re.search(r"cuda 12 queens result -1, calc time: \[", out)
    assert not ck.exists()


def test_resumable_rejects_foreign_or_broken_checkpoints(tmp_path):
    # Checked before any device work, so this runs without a GPU.
    import struct
    p = tmp_path / "ck"
    hdr = b"NQB200CK" + struct.pack("<IiiiqqQQq", 1, 10, 3, 0, 100, 5, 7, 1, 0)
    p.write_bytes(hdr)
    t = ctypes.c_uint64(0)
    d = ctypes.c_int(0)
    rc = nq.lib.nq_count_resumable(11, 3, None, str(p).encode(), ctypes.byref(t), ctypes.byref(d), None)
    assert rc == nq.NQ_ERR_ARG and "N=10" in nq.last_error()
    p.write_bytes(hdr[:-3])                                   # truncated
    assert nq.lib.nq_count_resumable(10, 3, None, str(p).encode(), ctypes.byref(t), ctypes.byref(d), None) \
        == nq.NQ_ERR_ARG
    p.write_bytes(b"XXXXXXXX" + hdr[8:])                      # wrong magic
    assert nq.lib.nq_count_resumable(10, 3, None, str(p).encode(), ctypes.byref(t), ctypes.byref(d), None) \
        == nq.NQ_ERR_ARG
    p.write_bytes(hdr + b"z")                                 # trailing bytes
    assert nq.lib.nq_count_resumable(10, 3, None, str(p).encode(), ctypes.byref(t), ctypes.byref(d), None) \
        == nq.NQ_ERR_ARG


def test_stack_levels_of_the_count_kernels():
    # The count step never enters rows N-2 and N-1, so it needs two stack slots
    # fewer than the node-counting step (which steps every row, like the
    # reference's loop with its STACKSIZE, src/macro.h:25-35); at least 1.
    assert nq.stack_levels(21, 6) == 12 and nq.stack_levels(21, 6, nodes=True) == 14
    assert nq.stack_levels(16, 5) == 8 and nq.stack_levels(4, 3) == 1
    with pytest.raises(nq.NQError):
        nq.stack_levels(40, 6)
