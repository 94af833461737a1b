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
