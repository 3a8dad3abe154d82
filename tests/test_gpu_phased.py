"""GPU parity of the phased-array path (yi-phasedarray, src/main.rs:2222-2412)
against the FP64 oracle: the phased power spectrum within the stated
tolerance, and the re-quantised phased .raw frames code-for-code except for
samples that lie within rounding distance of a decision boundary."""
import dataclasses

import numpy as np
import pytest

import oracle
from _cases import assert_spectra_close, make_scan, signal_raw, spectral_errors, to_fxc

pytestmark = pytest.mark.gpu


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def raw_codes(raw, n_samples, bits, shuffle):
    words = np.ascontiguousarray(raw).view("<u4").astype(np.uint32)
    words = oracle.np_shuffle_words(words, shuffle)
    per = 32 // bits
    sh = np.arange(per, dtype=np.uint32) * np.uint32(bits)
    codes = (words[:, None] >> sh[None, :]) & np.uint32((1 << bits) - 1)
    return codes.reshape(-1)[:n_samples]


def boundary_margin(x, levels):
    """Gap between the nearest and second-nearest level distance (f32)."""
    lv = np.asarray(levels, np.float32)
    err = np.sort(np.abs(x.astype(np.float32)[:, None] - lv[None, :]), axis=1)
    return err[:, 1] - err[:, 0]


CASES = [
    dict(fft=1024, grid=0, band=(5, 0, 507, 5), lsb1=True, lsb2=True),
    dict(fft=2048, grid=1, band=(-7, 7, 1024, 0), shuffle="generic", w1=0.7, w2=1.3),
    dict(fft=4096, grid=0, band=(40, 0, 2008, 40), shuffle="pairswap", lsb1=True),
    dict(fft=8192, grid=0, band=(-128, 128, 4096, 0), shuffle="generic", lsb1=True, lsb2=True),
    dict(fft=4096, bits1=2, bits2=4, grid=1, band=(12, 0, 2036, 12)),
    # FFT lengths above 8192: the two-row kernel (16384; 4- and 8-bit stations
    # staged in a row buffer), the cluster pair kernel (32768 / 65536 with the
    # band shift a multiple of N / 8192) and the four-step path (any other
    # shift, 4- and 8-bit stations)
    dict(fft=16384, grid=0, band=(-64, 64, 8192, 0), shuffle="generic", lsb1=True, lsb2=True),
    dict(fft=16384, bits1=4, bits2=2, grid=1, band=(32, 0, 8160, 32), shuffle="generic"),
    dict(fft=16384, bits1=8, bits2=8, grid=0, band=(-16, 16, 8192, 0), lsb1=True, lsb2=True),
    dict(fft=32768, bits1=1, bits2=2, grid=1, band=(100, 0, 16284, 100), w1=0.8, w2=1.2),
    dict(fft=65536, grid=0, band=(-64, 64, 32768, 0), shuffle="generic", lsb1=True, lsb2=True),
    dict(fft=32768, grid=1, band=(6, 0, 16378, 6), shuffle="pairswap"),
    dict(fft=32768, bits1=4, bits2=2, grid=0, band=(-32, 32, 16384, 0)),
]


@pytest.mark.parametrize("kw", CASES)
def test_phased_vs_fp64(engine, kw):
    delay = dict(net_d1_base=3.3e-7, total_rate1_base=2.1e-6, lo1_hz=8.4e9, lo2_hz=8.4e9,
                 net_d2_base=1.7e-8, total_rate2_base=-3e-7)
    scan = make_scan(fs=512e6, delay=delay, products=oracle.PROD_PHASED | oracle.PROD_RAW, **kw)
    nf = 40
    r1, r2 = signal_raw(scan, nf, seed=kw["fft"] + 3, rho=0.3, delay_samples=2.6)
    s = engine.open_scan(to_fxc(scan))
    got = s.sector_device(dev(r1), dev(r2), nf, first_frame=9)
    ref = oracle.fp64_sector_phased(scan, r1, r2, nf, first_frame=9)
    assert_spectra_close(got["phased"], ref["phased"], f"phased power {kw}")
    assert np.all(got["acf11"] == 0) and np.all(got["xcf"] == 0)

    n = scan.fft
    bo = scan.bits_out
    g = raw_codes(got["raw"], nf * n, bo, scan.shuffle1)
    x = ref["series"].reshape(-1)
    r = oracle.quantise_codes(x.astype(np.float32), scan.levels1)
    diff = g != r
    margin = boundary_margin(x, scan.levels1)
    scale = float(np.sqrt(np.mean(x ** 2)))
    assert diff.mean() < 1e-3, diff.mean()
    # every differing code sits on a decision boundary to f32 rounding
    assert np.all(margin[diff] < 1e-4 * scale), margin[diff].max()
    # The f32 restatement of the reference rotates each station with the
    # reference's f32 phase recurrence (utils.rs:115-117), which drifts ~1e-3 rad
    # across 4096 bins; its codes then differ from the GPU's on a slightly wider
    # band around the boundaries, so only the rate is bounded here.
    c = oracle.c_sector_phased(scan, r1, r2, nf, first_frame=9)
    cc = raw_codes(c["raw"], nf * n, bo, scan.shuffle1)
    assert (g != cc).mean() < 5e-3, (g != cc).mean()
    s.close()


def test_phased_host_path(engine):
    scan = make_scan(fft=4096, fs=512e6, band=(40, 0, 2008, 40), shuffle="generic",
                     delay=dict(net_d1_base=3.3e-7, lo1_hz=8.4e9, lo2_hz=8.4e9),
                     products=oracle.PROD_PHASED | oracle.PROD_RAW | oracle.PROD_ACF |
                     oracle.PROD_XCF)
    nf = 100
    r1, r2 = signal_raw(scan, nf, seed=4, rho=0.3)
    s = engine.open_scan(to_fxc(scan))
    a = s.sector_device(dev(r1), dev(r2), nf, first_frame=0)
    sid = s.submit(r1, r2, nf, 0)
    b = s.wait(sid)
    for k in ("acf11", "acf22", "xcf", "phased", "raw"):
        assert np.array_equal(a[k], b[k]), k
    assert np.any(a["acf11"]) and np.any(a["phased"])
    s.close()


@pytest.mark.parametrize("fft,lsb", [(4096, False), (8192, True), (16384, True), (65536, False)])
def test_phased_raw_round_trip(engine, fft, lsb):
    """The phased .raw decodes with the same plan (ant1's levels and shuffle,
    LSB when both inputs are LSB, src/main.rs:1093, 2391-2412) into a stream
    whose auto-spectrum is the phased power spectrum's shape: the GPU decode +
    ACF of the GPU-written frames equals the FP64 oracle's on the same bytes,
    and its normalised shape follows the phased power."""
    delay = dict(net_d1_base=2.1e-7, total_rate1_base=1.1e-6, lo1_hz=8.4e9, lo2_hz=8.4e9)
    scan = make_scan(fft=fft, fs=512e6, delay=delay, shuffle="generic", lsb1=lsb, lsb2=lsb,
                     products=oracle.PROD_PHASED | oracle.PROD_RAW, band=(0, 0, fft // 2, 0))
    nf = 120
    r1, r2 = signal_raw(scan, nf, seed=fft + 11, rho=0.6, delay_samples=1.5,
                        tone_bin=fft // 5)
    s = engine.open_scan(to_fxc(scan))
    ph = s.sector_device(dev(r1), dev(r2), nf, first_frame=0)
    s.close()
    raw = ph["raw"]
    # the round-trip scan: both "stations" are the phased stream, no delay
    rt = make_scan(fft=fft, fs=512e6, bits1=scan.bits_out, bits2=scan.bits_out,
                   levels1=list(scan.levels1), levels2=list(scan.levels1), shuffle="identity",
                   lsb1=lsb, lsb2=lsb, products=oracle.PROD_ACF, delay={})
    rt = dataclasses.replace(rt, shuffle1=list(scan.shuffle1), shuffle2=list(scan.shuffle1))
    s2 = engine.open_scan(to_fxc(rt))
    got = s2.sector_device(dev(raw), dev(raw), nf, first_frame=0)
    s2.close()
    ref = oracle.fp64_sector_corr(rt, raw, raw, nf, first_frame=0)
    assert_spectra_close(got["acf11"], ref["acf11"], "round-trip acf")
    # the second copy (overlap bins only) sees the same stream
    rel, _, _ = spectral_errors(got["acf22"][: fft // 2], got["acf11"][: fft // 2])
    assert rel < 1e-5, rel
    # shape: the re-quantised stream's spectrum follows the phased power
    a = got["acf11"][1:fft // 2] / np.mean(got["acf11"][1:fft // 2])
    p = ph["phased"][1:fft // 2] / np.mean(ph["phased"][1:fft // 2])
    assert np.corrcoef(a, p)[0, 1] > 0.9
    k = fft // 5  # the injected tone survives the round trip
    assert a[k - 1] > 1.8 * np.median(a) and p[k - 1] > 1.8 * np.median(p)
