import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


GPU = _gpu_available()


@pytest.fixture(scope="session")
def gpu():
    if not GPU:
        pytest.fail("GPU test collected on a machine without a CUDA device")
    return True


def need_ref(precision="double"):
    from oracle import ref
    if not ref.available(precision):
        pytest.skip("reference oracle library not built (make -C oracle)")
    return ref


def need_restated(precision="double"):
    from oracle import restated as rs
    if not rs.available(precision):
        pytest.skip("restatement not built (make -C oracle restate)")
    return rs
