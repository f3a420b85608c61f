import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ref():
    """The reference's own operators compiled against the oracle shims."""
    from oracle import refsim
    if not os.path.exists(refsim.LIB_PATH) and not os.path.isdir(refsim.REFERENCE_SOURCE):
        pytest.skip("oracle/_ref not built and reference sources absent")
    refsim.lib()
    return refsim
