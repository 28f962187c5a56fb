import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle and the engine library once per session (nvcc cross-compiles on CPU)."""
    from oracle import oracle
    oracle.build()
    if not os.environ.get("RT_SKIP_BUILD"):
        from renderlab_b200 import build
        build.build()
    yield


@pytest.fixture(scope="session")
def engine():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from renderlab_b200 import api
    e = api.Engine(0)
    yield e
    e.close()
