import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.fail("this test needs a CUDA device")
    return True


@pytest.fixture(scope="module")
def monkeypatch_module():
    """A monkeypatch that lives as long as a module-scoped fixture."""
    mp = pytest.MonkeyPatch()
    yield mp
    mp.undo()
