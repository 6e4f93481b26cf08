import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running full-size case")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


def golden_path(name):
    return os.path.join(GOLDEN, name)


def read_golden_elements(name):
    raw = open(golden_path(name), "rb").read()
    n = int(np.frombuffer(raw[:8], dtype="<u8")[0])
    return np.frombuffer(raw[8:], dtype="<u4", count=n).astype(np.uint32)


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch.device("cuda:0")
