"""fxc_sector_run_device_noalloc: the correlation call for callers that cannot
allocate device memory where they correlate (a real-time streaming loop that
must not stall the GPU on cudaMalloc/cudaFree's implicit synchronisation, or
an application whose memory manager owns all device memory).  Its scratch is
the library's fixed array, shared by every call.

Checked through the C ABI against the allocating entry point
(fxc_sector_run_device of an open scan) on two calls in a row with different
sectors, so a call that read state left by the previous one would show."""
import numpy as np
import pytest

import oracle
from _cases import assert_spectra_close, make_scan, signal_raw, to_fxc

pytestmark = pytest.mark.gpu


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("kw", [
    dict(fft=8192, fs=1024e6, shuffle="generic", lsb1=True, band=(-128, 128, 4096, 0)),
    dict(fft=1024, fs=32e6, bits1=4, bits2=2, band=(5, 0, 507, 5), grid=1,
         table=[1.0e-7, 1.2e-7, 1.4e-7]),
])
def test_noalloc_matches_allocating_entry_point(fxc_lib, kw):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    fxc = fxc_lib
    delay = dict(net_d1_base=3.3e-7, total_rate1_base=2.1e-6, lo1_hz=8.4e9, lo2_hz=8.416e9,
                 delay_user_samples=0.3)
    scan = make_scan(delay=delay, **kw)
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
        torch.cuda.synchronize()
        a = acc.cpu().numpy()
        got = dict(acf11=a[:h], acf22=a[h:2 * h], xcf=a[2 * h:4 * h].view(np.complex128))
        for k in ("acf11", "acf22", "xcf"):
            assert_spectra_close(got[k], ref[k], f"no-alloc call {call + 1} {k}")
        assert np.all(a[4 * h:] == 0)
    s.close()
    eng.close()


def test_noalloc_rejects_oversize(fxc_lib):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cfg = to_fxc(make_scan(fft=1024))
    d = torch.zeros(16, dtype=torch.uint8, device="cuda")
    acc = torch.zeros(5 * cfg.h, dtype=torch.float64, device="cuda")
    with pytest.raises(fxc_lib.FxcError, match="FXC_NOALLOC_MAX_FRAMES"):
        fxc_lib.sector_run_device_noalloc(cfg, d, d, fxc_lib.NOALLOC_MAX_FRAMES + 1, 0, acc)
    big = to_fxc(make_scan(fft=16384))
    with pytest.raises(fxc_lib.FxcError, match="fft_len above 8192"):
        fxc_lib.sector_run_device_noalloc(big, d, d, 1, 0, acc)
