"""Test configuration: the `gpu` marker and shared fixtures."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """A library context on cuda:0. GPU tests fail (not skip) without a GPU:
    they are only selected on a GPU box."""
    if not _cuda_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    from fbls_b200 import api
    g = api.Gpu(0)
    yield g
    g.close()
