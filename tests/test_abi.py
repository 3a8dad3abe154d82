"""C-ABI surface of libfxc.so, checked without a GPU: the library loads,
exports every function include/fxc.h declares, and its host helpers match
the known-answer vectors."""
import ctypes as C
import json
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
KAT = json.loads((Path(__file__).parent / "golden" / "kat.json").read_text())


def declared_functions():
    names = []
    for hdr in sorted((ROOT / "include").glob("*.h")):
        txt = hdr.read_text()
        names += re.findall(r"^FXC_API\s+[\w\s\*]+?\b(fxc_\w+)\s*\(", txt, flags=re.M)
    return names


def test_header_declares_functions():
    names = declared_functions()
    assert len(names) >= 20
    assert "fxc_sector_submit" in names and "fxc_sector_run_device" in names


def test_library_exports_every_declared_symbol(fxc_lib):
    lib = fxc_lib.lib()
    for n in declared_functions():
        assert hasattr(lib, n), f"libfxc.so does not export {n}"
    assert set(fxc_lib.EXPORTS) == set(declared_functions())
    assert lib.fxc_abi_version() == 1


def test_status_strings(fxc_lib):
    lib = fxc_lib.lib()
    for s in range(-8, 1):
        assert lib.fxc_status_string(s)


@pytest.mark.parametrize("case", KAT["parse_shuffle"])
def test_parse_shuffle(fxc_lib, case):
    if case["expect"] is None:
        with pytest.raises(fxc_lib.FxcError) as ei:
            fxc_lib.parse_shuffle(case["ext"])
        assert ei.value.status == fxc_lib.EINVAL
        assert "permutation" in str(ei.value)
    else:
        assert fxc_lib.parse_shuffle(case["ext"]) == case["expect"]


@pytest.mark.parametrize("case", KAT["band"])
def test_band_alignment(fxc_lib, case):
    args = (case["fft"], case["fs"], case["c1"], case["c2"], case["bw1"], case["bw2"])
    if case["expect"] is None:
        with pytest.raises(fxc_lib.FxcError, match="No band overlap"):
            fxc_lib.band_alignment(*args)
    else:
        assert list(fxc_lib.band_alignment(*args)) == case["expect"]


def test_level_power_and_normalize(fxc_lib):
    for c in KAT["level_power"]:
        assert fxc_lib.level_power(c["levels"]) == c["expect"]
    with pytest.raises(fxc_lib.FxcError):
        fxc_lib.level_power([0.0, 0.0])
    for c in KAT["normalize"]:
        out = fxc_lib.normalize(c["fft"], c["nf"], c["p"], acc_real=np.array(c["acc"]))
        np.testing.assert_allclose(out.real, c["expect"], rtol=1e-7)
    # the reference's own worked example (README.md:276-293)
    for c in KAT["readme"]["normalize"]:
        assert fxc_lib.level_power(c["levels"]) == c["p"]
        out = fxc_lib.normalize(c["fft"], c["nf"], c["p"], acc_real=np.array(c["acc"]))
        np.testing.assert_allclose(out.real, c["expect"], rtol=1e-7)


def test_normalize_matches_oracle(fxc_lib, oracle_lib):
    rng = np.random.default_rng(1)
    acc = rng.uniform(0, 1e9, 513)
    accc = rng.standard_normal(513) + 1j * rng.standard_normal(513)
    for kw in (dict(acc_real=acc), dict(acc_cplx=accc * 1e8)):
        a = fxc_lib.normalize(1024, 31250, 1.25, **kw)
        b = oracle_lib.c_normalize(1024, 31250, 1.25, **kw)
        np.testing.assert_array_equal(a, b)


def test_bytes_per_frame(fxc_lib):
    lib = fxc_lib.lib()
    assert lib.fxc_bytes_per_frame(8192, 2) == 2048
    assert lib.fxc_bytes_per_frame(1000, 3) == 375


def test_engine_create_without_gpu_fails_cleanly(fxc_lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(fxc_lib.FxcError):
        fxc_lib.Engine(0)
