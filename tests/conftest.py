import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the CUDA library and the oracle if their sources changed."""
    from behavert_b200 import build
    if os.environ.get("BRT_SKIP_BUILD") != "1":
        try:
            build.build_library()
        except Exception:
            if not build.LIB.exists():
                raise
        build.build_oracle()
    yield


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
