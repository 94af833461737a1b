"""Resumable counts (nq_count_resumable): a whole board counted in short
time slices with every interrupted lane's levels saved to a checkpoint file
and resumed must give the published total."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu


# The slices are short enough that some end before the lanes have taken every
# level the previous slice saved (those must carry over).
@pytest.mark.parametrize("N,k,slice_ms", [(17, 6, 1), (19, 6, 15), (18, 5, 4), (18, 6, 1)])
def test_sliced_count_is_exact(gpu, golden, tmp_path, N, k, slice_ms):
    ck = str(tmp_path / f"n{N}.ckpt")
    slices = 0
    while True:
        done, total, st = gpu.count_resumable(N, k, ck, slice_ms=slice_ms)
        slices += 1
        if done:
            break
        assert os.path.exists(ck) and not os.path.exists(ck + ".tmp")
        assert slices < 2000
    assert total == golden("published.json")[str(N)]["total"]
    assert slices > 2, slices           # the count really was interrupted and resumed
    assert not os.path.exists(ck)       # removed once the count finished


def test_unsliced_resumable_matches(gpu, golden, tmp_path):
    done, total, _ = gpu.count_resumable(16, 5, str(tmp_path / "x.ckpt"), slice_ms=0)
    assert done and total == golden("published.json")["16"]["total"]


def test_cli_checkpoint_mode(gpu, tmp_path):
    ck = str(tmp_path / "cli.ckpt")
    out = subprocess.run([gpu.CLI_PATH, "18", "6", "--checkpoint", ck, "--slice-ms", "5"], capture_output=True,
                         text=True, timeout=600).stdout
    assert "saved to" in out
    assert "cuda 18 queens result 666090624, calc time: [" in out
    assert not os.path.exists(ck)
