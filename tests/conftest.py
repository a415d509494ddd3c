import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "spid-join_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.lib()
    return o


@pytest.fixture(scope="session")
def spj():
    import spidjoin
    spidjoin.lib()
    return spidjoin


def main_cc_tables(n, ratio):
    """The reference driver's synthetic columns (test/join/main.cc:30-43)."""
    import numpy as np
    i = np.arange(n, dtype=np.uint64)
    R = np.stack([i + 1, i + 3], axis=1).astype(np.uint32)
    j = np.arange(n * ratio, dtype=np.uint64) // np.uint64(ratio)
    S = np.stack([j + 1, j + 3], axis=1).astype(np.uint32)
    return R, S
