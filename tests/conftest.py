"""pytest configuration: the `gpu` marker and import paths.

Tests marked gpu need a CUDA device and the built library; everything else
runs on CPU (oracle pins, host logic, ABI symbol checks)."""
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO / "hvd-cvbs-decoding_b200"))
sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and lib/libhvdg.so")


@pytest.fixture(scope="session")
def ctx():
    from hvdg import api
    c = api.Context(0)
    yield c
    c.close()
