import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "rust-wl_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: long CPU run (tens of seconds)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle.oracle as o
    o.load()
    return o


@pytest.fixture(scope="session")
def vxl():
    from vxl_sph import build as _b
    _b.build()
    import vxl_sph
    vxl_sph.load()
    return vxl_sph
