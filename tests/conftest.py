import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the CUDA path")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    for item in items:
        if "gpu" in item.keywords and not HAS_GPU:
            item.add_marker(pytest.mark.skip(reason="no CUDA device"))


@pytest.fixture(scope="session")
def ref_available():
    from oracle import psyref
    if not psyref.available():
        pytest.skip("oracle/_ref/libpsyref.so not built (make -C oracle ref)")
    return True


@pytest.fixture(scope="session")
def ctx():
    from psychopath_cpp_b200 import api
    c = api.Context(0)
    yield c
    c.close()
