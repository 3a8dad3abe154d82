import os
import shutil
import subprocess
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


@pytest.fixture(scope="session")
def tool(tmp_path_factory):
    """tests/cli_host_check.cpp built with the yi-* tools' host sources (no
    GPU library): run(command, *args) -> its stdout."""
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    cli = ROOT / "fx-corr_b200" / "cli"
    out = tmp_path_factory.mktemp("clihost") / "cli_host_check"
    srcs = [ROOT / "tests" / "cli_host_check.cpp"] + [cli / f for f in
                                                     ("args.cpp", "cor_writer.cpp", "geom.cpp",
                                                      "schedule.cpp")]
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", str(cli), *map(str, srcs), "-o", str(out)],
                   check=True, capture_output=True, text=True)

    def run(*args):
        r = subprocess.run([str(out), *map(str, args)], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0, r.stderr
        return r.stdout.strip()

    return run
