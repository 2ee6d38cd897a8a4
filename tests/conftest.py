import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the native libraries and the oracle once per session (no-ops when current)."""
    from harm_harm_b200 import build
    build.build_host()
    if not os.environ.get("HARM_SKIP_DEVICE_BUILD"):
        build.build_device()
    build.build_oracle()
    yield


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
