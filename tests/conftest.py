import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def built():
    """Builds liboctb.so and the oracle if needed (nvcc cross-compiles without a GPU)."""
    from octopusengine_b200.build import build
    build()
    import oracle_lib
    oracle_lib.lib()
    return True


@pytest.fixture(scope="session")
def ctx(built):
    import octopusengine_b200 as ob
    c = ob.Context(0, 8 << 30)
    yield c
    c.close()
