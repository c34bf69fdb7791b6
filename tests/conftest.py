import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def small_pair_np():
    """256 x 512 synthetic pair (same generator as the 1024 x 2048 workload)."""
    from specklesource_b200 import synth
    s1, s2 = synth.small_pair(na=256, nr=512)
    return synth.to_numpy(s1), synth.to_numpy(s2)
