import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def native_lib():
    from nanoshaper_b200 import build as nb
    nb.build()
    from nanoshaper_b200 import _native
    return _native.lib()


@pytest.fixture(scope="session")
def oracle_mod():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    O.build()
    return O
