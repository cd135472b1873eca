import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line(
        "markers", "slow: long CPU oracle runs; opt in with -m slow"
    )


def pytest_collection_modifyitems(config, items):
    expr = config.getoption("-m") or ""
    if "slow" in expr:
        return
    skip = pytest.mark.skip(reason="slow oracle run; select with -m slow")
    for item in items:
        if "slow" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
