import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


@pytest.fixture(scope="session")
def gpu_ready():
    """Skip-free GPU gate: on a GPU test the CUDA path must load and work."""
    from coherentsearch_c_b200.search import gpu_available
    rc, msg = gpu_available(0)
    assert rc == 1, f"B200 GPU required for -m gpu tests: {msg}"
    return msg
