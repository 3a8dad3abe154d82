"""fxc_sector_run_device_noalloc: the correlation call for callers that cannot
allocate device memory where they correlate (a real-time streaming loop that
must not stall the GPU on cudaMalloc/cudaFree's implicit synchronisation, or
an application whose memory manager owns all device memory).  Its scratch is
the library's fixed array, shared by every call.

Checked through the C ABI against the allocating entry point
(fxc_sector_run_device of an open scan) on two calls in a row with different
sectors, so a call that read state left by the previous one would show; the
first call is also held to the FP64 oracle.  Further cases: the device's free
memory does not change across calls, the layout's limits (the most frames per
call at FFT 8192, the longest geometric table), and a bounded wait that runs
out (fxc_debug_inject_wait_timeout) is reported by fxc_sector_noalloc_check
with NaN results, after which the next call is clean."""
import numpy as np
import pytest

import oracle
from _cases import assert_sector_close, assert_spectra_close, make_scan, signal_raw, to_fxc

pytestmark = pytest.mark.gpu

DELAY = dict(net_d1_base=3.3e-7, total_rate1_base=2.1e-6, lo1_hz=8.4e9, lo2_hz=8.416e9,
             delay_user_samples=0.3)


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def split(acc, h):
    a = acc.cpu().numpy()
    return dict(acf11=a[:h], acf22=a[h:2 * h], xcf=a[2 * h:4 * h].view(np.complex128)), a


def need_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("kw", [
    dict(fft=8192, fs=1024e6, shuffle="generic", lsb1=True, band=(-128, 128, 4096, 0)),
    dict(fft=1024, fs=32e6, bits1=4, bits2=2, band=(5, 0, 507, 5), grid=1,
         table=[1.0e-7, 1.2e-7, 1.4e-7]),
])
def test_noalloc_matches_allocating_entry_point(fxc_lib, kw):
    import torch

    need_gpu()
    fxc = fxc_lib
    scan = make_scan(delay=DELAY, **kw)
    cfg = to_fxc(scan)
    eng = fxc.Engine(0)
    s = eng.open_scan(cfg)
    h = cfg.h
    nf = 3000
    for call, (seed, first) in enumerate([(11, 0), (12, nf)]):
        r1, r2 = signal_raw(scan, nf, seed=seed, rho=0.1, delay_samples=3.3)
        d1, d2 = dev(r1), dev(r2)
        ref = s.sector_device(d1, d2, nf, first_frame=first)
        acc = torch.full((5 * h,), float("nan"), dtype=torch.float64, device="cuda")
        fxc.sector_run_device_noalloc(cfg, d1, d2, nf, first, acc)
        fxc.sector_noalloc_check()
        got, a = split(acc, h)
        for k in ("acf11", "acf22", "xcf"):
            assert_spectra_close(got[k], ref[k], f"no-alloc call {call + 1} {k}")
        assert np.all(a[4 * h:] == 0)
        if call == 0:
            fp = oracle.fp64_sector_corr(scan, r1, r2, nf, first_frame=first)
            assert_sector_close(got, fp, scan, "no-alloc vs fp64", nf=nf)
    s.close()
    eng.close()


def test_noalloc_allocates_nothing(fxc_lib):
    """After a first call (which looks up the array and loads the kernels),
    further calls leave the device's free memory exactly as it was."""
    import torch

    need_gpu()
    scan = make_scan(fft=8192, fs=1024e6, shuffle="generic", lsb1=True,
                     band=(128, 0, 3968, 128), delay=DELAY)
    cfg = to_fxc(scan)
    nf = 2000
    r1, r2 = oracle.synth_packed_pair(nf * 8192, 5, 2, scan.levels1, scan.shuffle1, True,
                                      scan.shuffle2, False, rho=0.1)
    d1, d2 = dev(r1), dev(r2)
    acc = torch.empty(5 * cfg.h, dtype=torch.float64, device="cuda")
    fxc_lib.sector_run_device_noalloc(cfg, d1, d2, nf, 0, acc)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for k in range(3):
        fxc_lib.sector_run_device_noalloc(cfg, d1, d2, nf, k * nf, acc)
        fxc_lib.sector_noalloc_check()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


@pytest.mark.parametrize("case", ["most_frames", "longest_table"])
def test_noalloc_at_its_limits(fxc_lib, case):
    import torch

    need_gpu()
    if case == "most_frames":  # fills the frame-record region of the array
        n, fs, nf = 8192, 1024e6, fxc_lib.NOALLOC_MAX_FRAMES
        table = 2.1e-7 - 0.5 / 8.4e9 * np.arange(3)
    else:  # fills the geometric-table slot beside the error word
        n, fs, nf = 1024, 32e6, 3000
        table = 1e-7 + 3e-9 * np.sin(np.arange(4096) / 300.0)
    scan = make_scan(fft=n, fs=fs, shuffle="generic", lsb1=True, band=(16, 0, n // 2 - 16, 16),
                     delay=dict(DELAY, delay_user_samples=0.0), table=table)
    cfg = to_fxc(scan)
    r1, r2 = oracle.synth_packed_pair(nf * n, 6, 2, scan.levels1, scan.shuffle1, True,
                                      scan.shuffle2, False, rho=0.1)
    d1, d2 = dev(r1), dev(r2)
    eng = fxc_lib.Engine(0)
    s = eng.open_scan(cfg)
    ref = s.sector_device(d1, d2, nf, first_frame=7)
    s.close()
    eng.close()
    acc = torch.empty(5 * cfg.h, dtype=torch.float64, device="cuda")
    fxc_lib.sector_run_device_noalloc(cfg, d1, d2, nf, 7, acc)
    fxc_lib.sector_noalloc_check()
    got, _ = split(acc, cfg.h)
    for k in ("acf11", "acf22", "xcf"):
        assert_spectra_close(got[k], ref[k], f"no-alloc {case} {k}")


def test_noalloc_reports_a_timed_out_wait(fxc_lib):
    import torch

    need_gpu()
    scan = make_scan(fft=8192, fs=1024e6, shuffle="generic", band=(128, 0, 3968, 128),
                     delay=DELAY)
    cfg = to_fxc(scan)
    nf = 500
    r1, r2 = oracle.synth_packed_pair(nf * 8192, 8, 2, scan.levels1, scan.shuffle1, False,
                                      scan.shuffle2, False, rho=0.1)
    d1, d2 = dev(r1), dev(r2)
    acc = torch.zeros(5 * cfg.h, dtype=torch.float64, device="cuda")
    try:
        fxc_lib.debug_inject_wait_timeout(256, True)
        fxc_lib.sector_run_device_noalloc(cfg, d1, d2, nf, 0, acc)
        with pytest.raises(fxc_lib.FxcError) as ei:
            fxc_lib.sector_noalloc_check()
        assert ei.value.status == fxc_lib.ETIMEDOUT
        assert torch.isnan(acc).all()
    finally:
        fxc_lib.debug_inject_wait_timeout(0, False)
    fxc_lib.sector_run_device_noalloc(cfg, d1, d2, nf, 0, acc)
    fxc_lib.sector_noalloc_check()
    got, _ = split(acc, cfg.h)
    ref = oracle.fp64_sector_corr(scan, r1, r2, nf)
    assert_sector_close(got, ref, scan, "no-alloc after an injected timeout", nf=nf)


def test_noalloc_rejects_oversize(fxc_lib):
    import torch

    need_gpu()
    cfg = to_fxc(make_scan(fft=1024))
    d = torch.zeros(16, dtype=torch.uint8, device="cuda")
    acc = torch.zeros(5 * cfg.h, dtype=torch.float64, device="cuda")
    with pytest.raises(fxc_lib.FxcError, match="FXC_NOALLOC_MAX_FRAMES"):
        fxc_lib.sector_run_device_noalloc(cfg, d, d, fxc_lib.NOALLOC_MAX_FRAMES + 1, 0, acc)
    big = to_fxc(make_scan(fft=16384))
    with pytest.raises(fxc_lib.FxcError, match="fft_len above 8192"):
        fxc_lib.sector_run_device_noalloc(big, d, d, 1, 0, acc)
    long_table = to_fxc(make_scan(fft=1024, table=np.zeros(4097)))
    with pytest.raises(fxc_lib.FxcError, match="FXC_NOALLOC_MAX_GEOM"):
        fxc_lib.sector_run_device_noalloc(long_table, d, d, 1, 0, acc)
