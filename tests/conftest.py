import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("dtv-net_b200", "oracle", os.path.join("tests", "golden")):
    p = os.path.join(REPO, sub)
    if p not in sys.path:
        sys.path.insert(0, p)
if REPO not in sys.path:  # bench.py, for the test of its FP64 check
    sys.path.append(REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built kernel library")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    return torch.device("cuda", 0)


def rel_rmse(a, b):
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.sqrt(np.mean((a - b) ** 2))
    n = np.sqrt(np.mean(b ** 2))
    return d / n if n > 0 else d
