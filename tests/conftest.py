import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    O.set_threads(1)  # deterministic summation order for parity
    return O


@pytest.fixture(scope="session")
def ctx():
    from nanotracer_b200 import CudaCtx
    c = CudaCtx(0)
    yield c
    c.close()
