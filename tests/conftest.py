import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    from tigerpm_b200 import _lib
    return _lib.load()


def pytest_collection_modifyitems(config, items):
    """Tests marked gpu are skipped, not failed, on a machine without CUDA."""
    if any("gpu" in item.keywords for item in items) and not has_gpu():
        skip = pytest.mark.skip(reason="needs a CUDA device")
        for item in items:
            if "gpu" in item.keywords:
                item.add_marker(skip)
