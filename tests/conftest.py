"""pytest configuration: the `gpu` marker and import paths for the package,
the oracle and the fixtures."""
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
for p in (REPO, REPO / "v1-1_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def built_lib():
    """Builds libsincgpu.so if it is missing or stale (nvcc cross-compiles on CPU)."""
    from sincgpu import _build
    return _build.build()
