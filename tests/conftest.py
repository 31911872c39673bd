import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests proper")


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not _has_gpu():
        pytest.skip("no CUDA device")
    import spice_b200

    spice_b200.library()  # the CUDA library must load; there is no fallback
    return True


@pytest.fixture(scope="session")
def oracle_built():
    import oracle

    if not os.path.exists(oracle.ORACLE_LIB):
        oracle.build(reference=False)
    return oracle
