import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the libqfb.so kernels)")
    config.addinivalue_line("markers", "slow: longer end-to-end runs")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


@pytest.fixture(scope="session")
def ref_qforte():
    """The compiled reference, where it can be imported (build container only)."""
    import warnings
    warnings.filterwarnings("ignore")
    from oracle import oracle as O
    try:
        return O.load_reference()
    except Exception as e:  # reference sources or module absent
        pytest.skip(f"reference not importable here: {e}")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
