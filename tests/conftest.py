import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


def _cuda_ok() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def femh():
    """The engine module; on a GPU box the library must load (no fallback)."""
    if not _cuda_ok():
        pytest.skip("no CUDA device")
    from fem_b200 import build
    build.build()
    import fem_b200
    fem_b200.load_library()
    return fem_b200
