"""GPU parity of the dihedral (8-fold) decomposition, through the C ABI.

Whole-board totals must equal the reference's (published totals, and the
oracle's plain total, which test_oracle.py pins to the reference); per-task
weighted counts must equal the oracle's restatement (oracle/dihedral_oracle.c)
bit for bit.
"""
import json
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
PUBLISHED = {int(k): v["total"] for k, v in json.load(open(os.path.join(GOLDEN, "published.json"))).items()}


def _known(N):
    return PUBLISHED[N] if N in PUBLISHED else oracle.total(N, 2)


def test_whole_board_small_n_every_depth(gpu):
    for N in range(4, 15):
        want = _known(N)
        for k in range(2, N - 1):
            r = gpu.count_dihedral(N, k)
            assert r.total == want, (N, k, r.total, want)


@pytest.mark.parametrize("N,k", [(15, 5), (16, 4), (16, 6), (17, 6), (18, 6), (19, 5), (19, 6), (20, 6), (20, 7)])
def test_whole_board_published(gpu, N, k):
    r = gpu.count_dihedral(N, k)
    assert r.total == PUBLISHED[N]
    assert r.stats["tasks"] == gpu.dihedral_expand(N, k)[0].size


@pytest.mark.parametrize("N,k", [(10, 3), (12, 4), (13, 5), (14, 5), (15, 5), (16, 6)])
def test_per_task_matches_oracle(gpu, N, k):
    c, l, r, cls, _ = gpu.dihedral_expand(N, k)
    got = gpu.count_dihedral_tasks(N, k, c, l, r, cls, per_task=True)
    want = oracle.dihedral_count_tasks(N, k, c, l, r, cls)
    assert np.array_equal(got["per_task"], want)
    assert got["sum"] == int(want.sum()) == _known(N)


def test_shuffled_mixed_classes(gpu):
    # Tasks of every class interleaved in the queue: lanes switch classes on
    # each refill, and in-warp donation hands class rules across lanes.
    N, k = 15, 5
    c, l, r, cls, _ = gpu.dihedral_expand(N, k)
    perm = np.random.default_rng(3).permutation(c.size)
    c, l, r, cls = c[perm], l[perm], r[perm], cls[perm]
    got = gpu.count_dihedral_tasks(N, k, c, l, r, cls, per_task=True,
                                   config={"block_threads": 64, "inner_steps": 8})
    want = oracle.dihedral_count_tasks(N, k, c, l, r, cls)
    assert np.array_equal(got["per_task"], want)
    # without donation, same result
    got2 = gpu.count_dihedral_tasks(N, k, c, l, r, cls, config={"steal": -1})
    assert got2["sum"] == _known(N)


def test_time_limit_reports_timeout(gpu):
    with pytest.raises(gpu.NQError) as e:
        gpu.count_dihedral(21, 6, config={"time_limit_ms": 2})
    assert e.value.status == gpu.NQ_ERR_TIMEOUT


def test_rejects_class_index_out_of_range(gpu):
    c, l, r, cls, classes = gpu.dihedral_expand(12, 4)
    bad = cls.copy()
    bad[0] = len(classes)
    with pytest.raises(gpu.NQError):
        gpu.count_dihedral_tasks(12, 4, c, l, r, bad)


def test_cli_dihedral(gpu):
    import re
    import subprocess
    exe = os.path.join(os.path.dirname(os.path.dirname(__file__)), "n_queens_b200", "n_queens")
    out = subprocess.run([exe, "16", "5", "--dihedral"], capture_output=True, text=True, timeout=120).stdout
    assert re.search(r"cuda 16 queens result 14772512, calc time", out), out


# Resumable dihedral counts: every saved level keeps its class, so the count
# is exact however often the kernel is stopped.
@pytest.mark.parametrize("N,k,slice_ms", [(16, 5, 1), (17, 6, 1), (18, 6, 3), (19, 7, 15)])
def test_sliced_dihedral_count_is_exact(gpu, tmp_path, N, k, slice_ms):
    ck = str(tmp_path / f"d{N}.ckpt")
    slices = 0
    while True:
        done, total, _ = gpu.count_resumable(N, k, ck, slice_ms=slice_ms, dihedral=True)
        slices += 1
        if done:
            break
        assert os.path.exists(ck) and not os.path.exists(ck + ".tmp")
        assert slices < 3000
    assert total == PUBLISHED[N]
    assert slices >= 2, slices          # interrupted at least once
    assert not os.path.exists(ck)


def test_dihedral_and_plain_checkpoints_do_not_mix(gpu, tmp_path):
    ck = str(tmp_path / "mix.ckpt")
    done, _, _ = gpu.count_resumable(18, 6, ck, slice_ms=2, dihedral=True)
    assert not done and os.path.exists(ck)
    with pytest.raises(gpu.NQError):
        gpu.count_resumable(18, 6, ck, slice_ms=2)
    while not done:
        done, total, _ = gpu.count_resumable(18, 6, ck, slice_ms=20, dihedral=True)
    assert total == PUBLISHED[18]


def test_cli_dihedral_checkpoint(gpu, tmp_path):
    import subprocess
    ck = str(tmp_path / "clid.ckpt")
    out = subprocess.run([gpu.CLI_PATH, "18", "6", "--dihedral", "--checkpoint", ck, "--slice-ms", "5"],
                         capture_output=True, text=True, timeout=600).stdout
    assert "saved to" in out
    assert "cuda 18 queens result 666090624, calc time: [" in out
    assert not os.path.exists(ck)


def test_checkpoint_with_bad_class_index_is_refused(gpu, tmp_path):
    ck = tmp_path / "bad.ckpt"
    done, _, _ = gpu.count_resumable(18, 6, str(ck), slice_ms=2, dihedral=True)
    assert not done
    raw = bytearray(ck.read_bytes())
    raw[-1] = 0xFF                       # the last saved level's class index
    ck.write_bytes(bytes(raw))
    with pytest.raises(gpu.NQError):
        gpu.count_resumable(18, 6, str(ck), slice_ms=2, dihedral=True)
    assert "class index" in gpu.last_error()


@pytest.mark.parametrize("cfg", [dict(block_threads=32), dict(block_threads=512), dict(layout=1), dict(steal=-1),
                                 dict(inner_steps=4), dict(inner_steps=8192), dict(stack_levels=25),
                                 dict(blocks_per_sm=1)])
def test_launch_shapes(gpu, cfg):
    assert gpu.count_dihedral(16, 5, config=cfg).total == PUBLISHED[16]
    assert gpu.count_dihedral(13, 3, config=cfg).total == PUBLISHED[13]
