import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "erdos-machine-13_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls the CUDA path through the C-ABI")
    config.addinivalue_line("markers", "slow: long parity case (tens of seconds)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def searches():
    import json
    with open(os.path.join(HERE, "golden", "searches.json")) as f:
        return {e["name"]: e for e in json.load(f)}
