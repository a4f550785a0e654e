import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords and not HAS_GPU:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def ref():
    import ref as refmod
    if not refmod.available():
        pytest.skip("reference build (oracle/_ref) not present")
    return refmod


@pytest.fixture(scope="session")
def ctx():
    import velox_b200
    c = velox_b200.Context(0)
    yield c
    c.close()
