"""Failure detection without a GPU fault.

The correlation kernels stage every frame through bulk copies tracked by
mbarriers whose waits are bounded.  fxc_debug_inject_wait_timeout makes those
waits run out on purpose: the kernels announce their copies but issue none,
so nothing is ever in flight, each CTA's first wait gives up after a few
hundred polls, the kernel records FXC_ETIMEDOUT in its error word and stops.
The host must see the error (fxc_scan_check, fxc_sector_wait), and the CUDA
context must stay usable: the next sector, with injection off, is correct.
"""
import time

import numpy as np
import pytest

import oracle
from _cases import assert_sector_close, make_scan, signal_raw, to_fxc

pytestmark = pytest.mark.gpu

DELAY = dict(net_d1_base=3.3e-7, total_rate1_base=2.1e-6, lo1_hz=8.4e9, lo2_hz=8.4e9)


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture
def injection(fxc_lib):
    yield fxc_lib.debug_inject_wait_timeout
    fxc_lib.debug_inject_wait_timeout(0, False)


# FFT 8192 and 16384 (even band shift): the fold kernels; 16384 with an odd
# band shift (2-bit stations): the one-CTA pair kernel; 65536 (a band shift
# that is a multiple of 8): the pair kernel, whose clusters' CTAs stop together
@pytest.mark.parametrize("fft,sb", [(8192, 128), (16384, 128), (16384, 129), (65536, 136)])
def test_bounded_wait_runs_out_and_is_reported(engine, fxc_lib, injection, fft, sb):
    scan = make_scan(fft=fft, fs=1024e6, shuffle="generic", lsb1=True,
                     band=(sb, 0, fft // 2 - sb, sb), delay=DELAY)
    nf = 600
    r1, r2 = signal_raw(scan, nf, seed=21, rho=0.2, delay_samples=3.3)
    d1, d2 = dev(r1), dev(r2)
    s = engine.open_scan(to_fxc(scan))
    times = {}
    for polls in (256, 2048):
        injection(polls, True)
        t0 = time.perf_counter()
        with pytest.raises(fxc_lib.FxcError) as ei:
            s.sector_device(d1, d2, nf)  # runs, then fxc_scan_check
        times[polls] = time.perf_counter() - t0
        assert ei.value.status == fxc_lib.ETIMEDOUT, ei.value
    injection(0, False)
    # the context is usable and the error word was cleared: a clean sector
    got = s.sector_device(d1, d2, nf)
    ref = oracle.fp64_sector_corr(scan, r1, r2, nf)
    assert_sector_close(got, ref, scan, f"after injected timeouts fft={fft}", nf=nf)
    s.close()
    print(f"injected timeouts fft={fft}: 256 polls {times[256] * 1e3:.1f} ms, "
          f"2048 polls {times[2048] * 1e3:.1f} ms")


def test_sector_wait_reports_timeout(engine, fxc_lib, injection):
    """The host-buffer path: fxc_sector_wait returns FXC_ETIMEDOUT for the
    sector whose kernel gave up, and the next sector on the scan is clean."""
    scan = make_scan(fft=8192, fs=1024e6, shuffle="generic", band=(128, 0, 3968, 128),
                     delay=DELAY)
    nf = 300
    r1, r2 = signal_raw(scan, nf, seed=22, rho=0.2)
    s = engine.open_scan(to_fxc(scan))
    injection(512, True)
    sid = s.submit(r1, r2, nf, 0)
    with pytest.raises(fxc_lib.FxcError) as ei:
        s.wait(sid)
    assert ei.value.status == fxc_lib.ETIMEDOUT
    injection(0, False)
    got = s.wait(s.submit(r1, r2, nf, 0))
    ref = oracle.fp64_sector_corr(scan, r1, r2, nf)
    assert_sector_close(got, ref, scan, "sector after an injected timeout", nf=nf)
    s.close()
