"""Shared test setup: marker registration, import path, in-tree builds."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the product library and the oracles once per session."""
    import cipher_b200.build as b
    import oracle
    try:
        b.build()
    except RuntimeError:
        # the GPU box has no need to rebuild when the prebuilt library is present
        if not os.path.exists(b.LIB):
            raise
    oracle.build(ref=True)
    yield


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
