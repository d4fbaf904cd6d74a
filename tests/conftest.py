import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The library a test gets when it names none is the exact build, whatever
# GFX_FLUID_VARIANT says: the bit-level and per-field parity claims are that
# build's.  The tests of the fast build name it (variant="fast") and assert
# its own bar, 1e-12 of each quantity per step.
os.environ["GFX_FLUID_VARIANT"] = "exact"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
