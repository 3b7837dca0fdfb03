import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build (or reuse) the in-tree native libraries once per session."""
    from fdmap_github_b200.build import build_library
    from oracle.build import build_oracle

    if os.environ.get("FDMAP_SKIP_BUILD") != "1":
        build_library()
    build_oracle()
    yield


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture
def require_gpu():
    if not gpu_available():
        pytest.fail("this test is marked gpu and needs a CUDA device")
