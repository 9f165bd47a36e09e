import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the fused kernels")


@pytest.fixture(scope="session")
def golden():
    """Golden vectors recorded from the reference build (tests/golden/make_golden.py)."""
    import json

    import numpy as np
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        index = json.load(f)
    arrays = np.load(os.path.join(ROOT, "tests", "golden", "golden.npz"))
    return index, arrays


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return torch.device("cuda", 0)
