import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")


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


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle and the CUDA library once per session (no-ops when current)."""
    from oracle.build import build_oracle

    build_oracle()
    from ifgf_b200 import build as b

    b.build()
