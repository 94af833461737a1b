"""The batched workload: 4096 uneven partial boards (N in [12,20], m in
[0,4], seed 1) in one launch, each count against the reference's."""
import os

import pytest

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "boards_4096.json")


def test_batch_4096_matches_reference(gpu, golden):
    g = golden("boards_4096.json")
    inst = [tuple(b) for b in g["instances"]]
    out = gpu.count_batch(inst)
    assert out.tolist() == g["counts"]
