import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libcintx_cuda.so")


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_cuda():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def close(a, b, atol=1e-12, rtol=1e-10):
    """Reference parity rule: |d| <= atol or |d| <= rtol*|ref| per element
    (cintx-oracle tests/two_electron_parity.rs:26-33)."""
    import numpy as np
    d = np.abs(np.asarray(a) - np.asarray(b))
    return bool(np.all((d <= atol) | (d <= rtol * np.abs(b))))
