"""Parity at the workloads' full sizes, through the C ABI.

* The full-rate plain workload (1024 Msps, 2-bit, FFT 8192, generic shuffle,
  station 1 LSB / station 2 USB, 16 MHz band offset, geometric table with a
  0.5 Hz fringe, residual delay 0.3 samples and rate 0.01 Hz): one whole
  1-s sector of 125000 frame pairs against the C restatement of the reference
  path on the same bytes, and its first 31250 frame pairs against the FP64
  oracle, which also states the restatement's own drift from FP64.
* The precision sweep's 2-s scans at 512 Msps (1.024e9 samples per station,
  rho = 0.01 plus a -30 dB tone), FFT 1024 (1e6 frames) and 65536, whole,
  against the FP64 oracle: the kernels accumulate up to 32 frames in f32
  registers before adding them to f64 partials, checked here over 1e6 frames.
"""
import numpy as np
import pytest

import oracle
from _cases import (REL_AMP_TOL, assert_sector_close, make_scan, spectral_errors, to_fxc,
                    xcf_drift_bound, xcf_floor)

pytestmark = pytest.mark.gpu


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_full_rate_sector_vs_restatement_and_fp64(engine):
    import bench

    scan = bench.oracle_scan()
    n, nf, sector = scan.fft, bench.NF_SECTOR, 3
    first = sector * nf  # table interpolation between seconds 3 and 4
    r1, r2 = oracle.synth_packed_pair(nf * n, 4242, 2, scan.levels1, scan.shuffle1, scan.lsb1,
                                      scan.shuffle2, scan.lsb2, rho=bench.RHO, lag=7)
    d1, d2 = dev(r1), dev(r2)
    s = engine.open_scan(to_fxc(scan))
    got = s.sector_device(d1, d2, nf, first_frame=first)
    c = oracle.c_sector_corr(scan, r1, r2, nf, first_frame=first)
    assert c["failed"] == 0
    _, a1s, a1e, _ = scan.band
    bound = xcf_drift_bound(a1e - a1s)
    # the whole sector against the restatement on the same bytes
    for k in ("acf11", "acf22"):
        rel, ph, ab = spectral_errors(got[k], c[k])
        assert rel <= REL_AMP_TOL and ab <= REL_AMP_TOL, (k, rel, ab)
    rel, ph, ab = spectral_errors(got["xcf"], c["xcf"], xcf_floor(c, nf))
    assert rel <= bound["rel_amp"] and ph <= bound["phase_rad"], (rel, ph, bound)
    # a quarter sector against FP64: the GPU within the stated tolerance, the
    # restatement within its recurrence's drift bound
    m = nf // 4
    b = scan.bpf(2)
    g_s = s.sector_device(d1[:m * b], d2[:m * b], m, first_frame=first)
    s.close()
    ref = oracle.fp64_sector_corr_parallel(scan, r1[:m * b], r2[:m * b], m, first_frame=first)
    assert_sector_close(g_s, ref, scan, "full-rate quarter sector vs fp64", nf=m)
    c_s = oracle.c_sector_corr(scan, r1[:m * b], r2[:m * b], m, first_frame=first)
    rel, ph, ab = spectral_errors(c_s["xcf"], ref["xcf"], xcf_floor(ref, m))
    assert rel <= bound["rel_amp"] and ph <= bound["phase_rad"], (rel, ph, bound)
    for k in ("acf11", "acf22"):
        assert spectral_errors(c_s[k], ref[k])[0] <= REL_AMP_TOL


@pytest.mark.parametrize("fft", [1024, 65536])
def test_two_second_scan_vs_fp64(engine, fft):
    fs, seconds = 512e6, 2.0
    nf = int(seconds * fs) // fft
    rng = np.random.Generator(np.random.PCG64(fft + 3))
    tone = int(rng.integers(fft // 16, fft // 2 - fft // 16))
    sb = 16 * fft // 1024
    delay = dict(net_d1_base=3.3e-7, total_rate1_base=2.1e-6, lo1_hz=8.4e9, lo2_hz=8.4e9)
    scan = make_scan(fft=fft, fs=fs, bits1=2, bits2=2, shuffle="generic", lsb1=True,
                     band=(sb, 0, fft // 2 - sb, sb), delay=delay)
    r1, r2 = oracle.synth_packed_pair(nf * fft, fft, 2, scan.levels1, scan.shuffle1, True,
                                      scan.shuffle2, False, rho=0.01, lag=4, tone_bin=tone,
                                      fft=fft)
    s = engine.open_scan(to_fxc(scan))
    got = s.sector_device(dev(r1), dev(r2), nf, first_frame=0)
    s.close()
    ref = oracle.fp64_sector_corr_parallel(scan, r1, r2, nf)
    assert_sector_close(got, ref, scan, f"2-s scan fft={fft} nf={nf}", nf=nf)
    a = got["acf11"]
    med = float(np.median(a[1:fft // 2]))
    assert a[tone] - med > 5 * med / np.sqrt(nf)
