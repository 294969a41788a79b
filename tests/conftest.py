import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (runs through the C-ABI)")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def renderer():
    """One GPU context for the session.  Fails (not skips) without a GPU: the
    gpu-marked tests are only selected where a GPU exists."""
    from blackhole_b200 import Renderer

    r = Renderer(0)
    yield r
    r.close()


@pytest.fixture(scope="session")
def orc():
    import oracle

    return oracle.oracle()


@pytest.fixture(scope="session")
def ref():
    import oracle

    port = oracle.reference()
    if port is None:
        pytest.skip("the reference harness oracle/_ref was not built here")
    return port
