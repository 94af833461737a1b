import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (a B200); run with -m gpu")


@pytest.fixture(scope="session")
def golden():
    import json

    def load(name):
        with open(os.path.join(GOLDEN, name)) as f:
            return json.load(f)

    return load


@pytest.fixture(scope="session")
def gpu():
    """The library, after checking that a CUDA device is present (fails, never skips)."""
    import n_queens_b200 as nq

    assert nq.device_count() > 0, "GPU tests need a CUDA device"
    return nq
