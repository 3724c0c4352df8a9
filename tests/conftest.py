import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libvsjoin.so")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def vsabi():
    from vibespatial_b200 import _abi

    _abi.load()
    return _abi


@pytest.fixture(scope="session")
def ctx(vsabi):
    return vsabi.default_context(0)
