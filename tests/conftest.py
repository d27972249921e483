import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")
    # build (or find current) the CUDA library and the oracle before the test
    # modules are collected: they import the package, which needs the library
    import __graft_entry__

    __graft_entry__.build()


_HAS_GPU = None


def has_gpu():
    global _HAS_GPU
    if _HAS_GPU is None:
        try:
            import torch

            _HAS_GPU = torch.cuda.is_available()
        except Exception:
            _HAS_GPU = False
    return _HAS_GPU


def pytest_collection_modifyitems(config, items):
    for item in items:
        if "gpu" in item.keywords and not has_gpu():
            item.add_marker(pytest.mark.skip(reason="no CUDA device visible"))
