"""Precision sweep: bit depths 1/2/4/8 x FFT
1024/4096/16384/65536 at 512 Msps, correlated noise at rho = 0.01 plus a
-30 dB tone at a seeded channel; the FP32 GPU path against the FP64 oracle,
amplitude and phase error per bin.  Each case runs a bounded sample of the
2-s scan (about 4 M samples per station) so the FP64 oracle stays quick; the
errors per bin do not depend on the scan length once the cross-station leak
cancels (test_gpu_parity.py::test_weak_correlation_long_integration; the
whole 2-s scans of FFT 1024 and 65536 run in test_gpu_full_size.py).

Every case also states the C restatement of the reference path against the
same FP64 oracle, whose f32 phase-ramp recurrence drifts by up to
ov * 2^-23 (tests/_cases.py xcf_drift_bound), and the GPU against that
restatement; with FXC_SWEEP_LOG set each case appends one JSON line with
the three sets of errors (the drift table).  test_drift_configs adds the
plain workloads at FFT 1024 (32 Msps) and FFT 8192 (1024 Msps)."""
import json
import os

import numpy as np
import pytest

import oracle
from _cases import (PHASE_TOL, REL_AMP_TOL, assert_sector_close, make_scan, signal_raw,
                    spectral_errors, to_fxc, xcf_drift_bound, xcf_floor)

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
    log_case(dict(workload="sweep", bits=bits, fft=fft, frames=nf, tone_bin=tone), scan, r1, r2,
             nf, 3, got, ref, out)


NAMES = ("rel_amp", "phase_rad", "abs_rms")


def log_case(head, scan, r1, r2, nf, first, got, ref, gpu_errs):
    """Restatement vs FP64 and GPU vs restatement beside GPU vs FP64; checks
    the restatement's drift against its bound and the GPU against the
    restatement within that drift plus the GPU tolerance; appends the table
    line to $FXC_SWEEP_LOG."""
    c = oracle.c_sector_corr(scan, r1, r2, nf, first_frame=first)
    fl = xcf_floor(ref, nf)
    drift = {k: spectral_errors(c[k], ref[k], fl if k == "xcf" else None)
             for k in ("acf11", "acf22", "xcf")}
    g_c = {k: spectral_errors(got[k], c[k], fl if k == "xcf" else None)
           for k in ("acf11", "acf22", "xcf")}
    _, a1s, a1e, _ = scan.band_or_default()
    bound = xcf_drift_bound(a1e - a1s)
    assert drift["xcf"][0] <= bound["rel_amp"] and drift["xcf"][1] <= bound["phase_rad"], drift
    assert g_c["xcf"][0] <= 1.01 * drift["xcf"][0] + REL_AMP_TOL, (g_c, drift)
    assert g_c["xcf"][1] <= 1.01 * drift["xcf"][1] + PHASE_TOL, (g_c, drift)
    line = dict(head, overlap_bins=a1e - a1s,
                **{f"gpu_fp64_{k}_{m}": float(v) for k, r in gpu_errs.items()
                   for m, v in zip(NAMES, r)},
                **{f"ref_fp64_{k}_{m}": float(v) for k, r in drift.items()
                   for m, v in zip(NAMES, r)},
                **{f"gpu_ref_{k}_{m}": float(v) for k, r in g_c.items()
                   for m, v in zip(NAMES, r)},
                xcf_bound_rel_amp=bound["rel_amp"], xcf_bound_phase=bound["phase_rad"])
    path = os.environ.get("FXC_SWEEP_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(line) + "\n")


@pytest.mark.parametrize("which", ["fft1024_32msps", "fft8192_1024msps"])
def test_drift_configs(engine, which):
    """The plain workloads' shapes: FFT 1024 at 32 Msps (rho = 0.05, the
    123.4-sample lag, identity shuffle, USB) and the full-rate FFT 8192 scan
    (generic shuffle, LSB/USB, 16 MHz band offset, 0.5 Hz fringe, residual
    delay and rate) on a 4000-frame slice of its fourth second."""
    import torch

    import bench

    if which == "fft1024_32msps":
        scan = make_scan(fft=1024, fs=32e6, delay=dict(net_d1_base=1.5e-6 - 48 / 32e6,
                                                         total_rate1_base=1e-12, d_seek=48 / 32e6,
                                                         lo1_hz=8.4e9, lo2_hz=8.4e9))
        nf, first = 4000, 0
        r1, r2 = signal_raw(scan, nf, seed=11, rho=0.05, delay_samples=123.4)
    else:
        scan = bench.oracle_scan()
        nf, first = 4000, 3 * bench.NF_SECTOR
        r1, r2 = oracle.synth_packed_pair(nf * scan.fft, 77, 2, scan.levels1, scan.shuffle1,
                                          scan.lsb1, scan.shuffle2, scan.lsb2, rho=bench.RHO)
    s = engine.open_scan(to_fxc(scan))
    got = s.sector_device(torch.from_numpy(r1).cuda(), torch.from_numpy(r2).cuda(), nf,
                          first_frame=first)
    s.close()
    ref = oracle.fp64_sector_corr(scan, r1, r2, nf, first_frame=first)
    out = assert_sector_close(got, ref, scan, which, nf=nf, ref_acf=ref)
    log_case(dict(workload=which, bits=2, fft=scan.fft, frames=nf), scan, r1, r2, nf, first, got,
             ref, out)
