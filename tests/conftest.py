import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT / "fx-corr_b200", ROOT / "oracle", ROOT / "tests", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def fxc_lib():
    import fxc
    from fxc import build as fxc_build

    if not fxc.LIB_PATH.exists():
        fxc_build.build()
    fxc.lib()
    return fxc


@pytest.fixture(scope="session")
def engine(fxc_lib):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eng = fxc_lib.Engine(0, max_inflight=3)
    yield eng
    eng.close()
