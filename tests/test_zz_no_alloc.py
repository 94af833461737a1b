"""The allocation-free device entry, nq_count_tasks_device_noalloc.

It is for callers that cannot let the library call cudaMalloc (a framework
whose allocator owns the GPU's memory, a service that forbids allocation after
start-up): its scratch sits in a fixed array inside the library.  This file
runs last (pytest collects it after every other test file) and checks the new
entry through the C ABI against nq_count_tasks_device, the entry that keeps
its scratch in library-allocated memory, on two calls in a row -- the second
call must not see what the first left in the shared array.
"""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _device_tasks(torch, N, k):
    c, l, r = oracle.expand(N, k)
    dev = torch.device("cuda:0")
    to = lambda a: torch.from_numpy(a.view(np.int32)).to(dev)
    return c.size, to(c), to(l), to(r)


def _run(gpu, fn, N, n, tc, tl, tr, out, cfg, stream):
    rc = fn(N, tc.data_ptr(), tl.data_ptr(), tr.data_ptr(), n, out.data_ptr(), ctypes.byref(cfg),
            stream.cuda_stream)
    assert rc == 0, (rc, gpu.last_error())


def test_noalloc_matches_allocating_entry_twice(gpu):
    import torch
    stream = torch.cuda.current_stream()
    for N, k in [(16, 5), (17, 6)]:
        n, tc, tl, tr = _device_tasks(torch, N, k)
        cfg = gpu.Config()
        cfg.stack_levels = N - 1 - k
        want = torch.zeros(2, dtype=torch.int64, device="cuda:0")
        rc = gpu.lib.nq_count_tasks_device(N, tc.data_ptr(), tl.data_ptr(), tr.data_ptr(), n, None, None,
                                           want.data_ptr(), ctypes.byref(cfg), stream.cuda_stream)
        assert rc == 0
        for _ in range(2):
            got = torch.full((2,), -7, dtype=torch.int64, device="cuda:0")
            _run(gpu, gpu.lib.nq_count_tasks_device_noalloc, N, n, tc, tl, tr, got, cfg, stream)
            torch.cuda.synchronize()
            assert got.tolist() == want.tolist(), (N, k)
        assert int(want[1]) == 0
        assert 2 * int(want[0]) == oracle.total(N, k)


def test_noalloc_rejects_grid_beyond_its_array(gpu):
    import torch
    n, tc, tl, tr = _device_tasks(torch, 10, 3)
    cfg = gpu.Config()
    cfg.blocks_per_sm = 1000  # x SMs is far beyond the array's CTA slots
    out = torch.zeros(2, dtype=torch.int64, device="cuda:0")
    rc = gpu.lib.nq_count_tasks_device_noalloc(10, tc.data_ptr(), tl.data_ptr(), tr.data_ptr(), n,
                                               out.data_ptr(), ctypes.byref(cfg),
                                               torch.cuda.current_stream().cuda_stream)
    assert rc == gpu.NQ_ERR_ARG
    assert "scratch array" in gpu.last_error()


def test_noalloc_status_word_does_not_leak_into_the_next_call(gpu):
    # A call whose tasks need more stack levels than it was given sets the
    # depth bit (1) of its status word; the next, correct call on the same
    # shared array must report status 0 and the allocating entry's sum.
    import torch
    stream = torch.cuda.current_stream()
    N, k = 15, 5
    n, tc, tl, tr = _device_tasks(torch, N, k)
    bad = gpu.Config()
    bad.stack_levels = 1  # far fewer slots than these tasks need
    got = torch.full((2,), -7, dtype=torch.int64, device="cuda:0")
    _run(gpu, gpu.lib.nq_count_tasks_device_noalloc, N, n, tc, tl, tr, got, bad, stream)
    torch.cuda.synchronize()
    assert int(got[1]) & 1
    good = gpu.Config()
    good.stack_levels = N - 1 - k
    want = torch.zeros(2, dtype=torch.int64, device="cuda:0")
    rc = gpu.lib.nq_count_tasks_device(N, tc.data_ptr(), tl.data_ptr(), tr.data_ptr(), n, None, None,
                                       want.data_ptr(), ctypes.byref(good), stream.cuda_stream)
    assert rc == 0
    _run(gpu, gpu.lib.nq_count_tasks_device_noalloc, N, n, tc, tl, tr, got, good, stream)
    torch.cuda.synchronize()
    assert int(got[1]) == 0
    assert got.tolist() == want.tolist()
    assert 2 * int(got[0]) == oracle.total(N, k)


def test_noalloc_runs_the_allocating_entrys_launch_shape(gpu, golden):
    # Both entries pick the CTA size and queue chunking the same way, so at
    # the N=19, k=6 whole board they count the same total in about the same
    # time (kernel time per entry, CUDA events on the launching stream).
    import torch
    stream = torch.cuda.current_stream()
    N, k = 19, 6
    c, l, r = gpu.expand(N, k)
    dev = torch.device("cuda:0")
    tc, tl, tr = (torch.from_numpy(a.view(np.int32)).to(dev) for a in (c, l, r))
    cfg = gpu.Config()
    cfg.stack_levels = N - 1 - k
    outs, ms = {}, {}
    for name in ("nq_count_tasks_device", "nq_count_tasks_device_noalloc", "nq_count_tasks_device",
                 "nq_count_tasks_device_noalloc"):
        fn = getattr(gpu.lib, name)
        out = torch.full((2,), -7, dtype=torch.int64, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if name.endswith("noalloc"):
            rc = fn(N, tc.data_ptr(), tl.data_ptr(), tr.data_ptr(), c.size, out.data_ptr(), ctypes.byref(cfg),
                    stream.cuda_stream)
        else:
            rc = fn(N, tc.data_ptr(), tl.data_ptr(), tr.data_ptr(), c.size, None, None, out.data_ptr(),
                    ctypes.byref(cfg), stream.cuda_stream)
        assert rc == 0, gpu.last_error()
        e1.record(stream)
        torch.cuda.synchronize()
        outs.setdefault(name, []).append(out.tolist())
        ms.setdefault(name, []).append(e0.elapsed_time(e1))
    want = golden("published.json")[str(N)]["total"]
    for name, vals in outs.items():
        for v in vals:
            assert 2 * v[0] == want and v[1] == 0, (name, v)
    a, b = min(ms["nq_count_tasks_device"]), min(ms["nq_count_tasks_device_noalloc"])
    print(f"N={N} k={k}: allocating entry {a:.1f} ms, allocation-free entry {b:.1f} ms")
    assert b <= 1.05 * a

