import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the native libraries and the oracle once per session if they are missing or stale."""
    from oracle import oracle
    from polysolve_b200 import _build

    _build.build_syn()
    _build.build_mas()
    oracle.build()
    yield
