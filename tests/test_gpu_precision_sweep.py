"""Precision sweep: bit depths 1/2/4/8 x FFT
1024/4096/16384/65536 at 512 Msps, correlated noise at rho = 0.01 plus a
-30 dB tone at a seeded channel; the FP32 GPU path against the FP64 oracle,
amplitude and phase error per bin.  Each case runs a bounded sample of the
2-s scan (about 4 M samples per station) so the FP64 oracle stays quick; the
errors per bin do not depend on the scan length once the cross-station leak
cancels (test_gpu_parity.py::test_weak_correlation_long_integration)."""
import json
import os

import numpy as np
import pytest

import oracle
from _cases import assert_sector_close, make_scan, signal_raw, spectral_errors, to_fxc, xcf_floor

pytestmark = pytest.mark.gpu

DELAY = dict(net_d1_base=3.3e-7, total_rate1_base=2.1e-6, lo1_hz=8.4e9, lo2_hz=8.4e9)


@pytest.mark.parametrize("fft", [1024, 4096, 16384, 65536])
@pytest.mark.parametrize("bits", [1, 2, 4, 8])
def test_precision_sweep(engine, bits, fft):
    import torch

    nf = max(8, (1 << 22) // fft)
    rng = np.random.Generator(np.random.PCG64(bits * 100003 + fft))
    tone = int(rng.integers(fft // 16, fft // 2 - fft // 16))
    sb = 16 * fft // 1024
    scan = make_scan(fft=fft, fs=512e6, bits1=bits, bits2=bits, shuffle="generic", lsb1=True,
                     band=(sb, 0, fft // 2 - sb, sb), delay=DELAY)
    r1, r2 = signal_raw(scan, nf, seed=fft + bits, rho=0.01, delay_samples=4.2, tone_bin=tone)
    s = engine.open_scan(to_fxc(scan))
    got = s.sector_device(torch.from_numpy(r1).cuda(), torch.from_numpy(r2).cuda(), nf,
                          first_frame=3)
    s.close()
    ref = oracle.fp64_sector_corr(scan, r1, r2, nf, first_frame=3)
    out = assert_sector_close(got, ref, scan, f"sweep bits={bits} fft={fft}", nf=nf, ref_acf=ref)
    # the tone stands out of the auto-spectrum (5 sigma of the per-bin noise)
    a = got["acf11"]
    med = float(np.median(a[1:fft // 2]))
    assert a[tone] - med > 5 * med / np.sqrt(nf), (a[tone] / med, nf)
    line = dict(bits=bits, fft=fft, frames=nf, tone_bin=tone,
                **{f"{k}_{m}": float(v) for k, r in out.items()
                   for m, v in zip(("rel_amp", "phase_rad", "abs_rms"), r)})
    path = os.environ.get("FXC_SWEEP_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(line) + "\n")
