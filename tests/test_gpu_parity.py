"""GPU parity of the sm_100a path, called through the C ABI, against the
oracle: decode + integer shift and the delay model bit-exact; spectra and
sector accumulators within the stated tolerance of the FP64 oracle."""
import dataclasses
import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
from _cases import (PHASE_TOL, REL_AMP_TOL, assert_sector_close, assert_spectra_close,
                    make_scan, random_raw, signal_raw, spectral_errors, to_fxc, xcf_drift_bound,
                    xcf_floor)

pytestmark = pytest.mark.gpu
KAT = json.loads((Path(__file__).parent / "golden" / "kat.json").read_text())

DELAY = dict(net_d1_base=3.3e-7, total_rate1_base=2.1e-6, lo1_hz=8.4e9, lo2_hz=8.4e9)


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


# ------------------------------------------------------------ decode + shift

DECODE_CASES = [(n, b, sh, l1, l2) for n in (1024, 8192) for b in (1, 2, 4, 8)
                for sh in ("identity", "pairswap", "generic") for (l1, l2) in ((False, True),)]
DECODE_CASES += [(2048, 2, "generic", True, True), (4096, 2, "identity", False, False),
                 (8192, 2, "sample2", True, False), (8192, 2, "generic", True, True)]


@pytest.mark.parametrize("n,bits,sh,l1,l2", DECODE_CASES)
def test_decode_shift_bit_exact(engine, n, bits, sh, l1, l2):
    # a delay model that sweeps integer shifts through +-N and beyond
    fs = 32e6
    delay = dict(net_d1_base=-1.3 * n / fs, total_rate1_base=2.7 * n / fs / (40 * n / fs),
                 net_d2_base=5.0 / fs, total_rate2_base=-0.05)
    scan = make_scan(fft=n, fs=fs, bits1=bits, bits2=bits, shuffle=sh, lsb1=l1, lsb2=l2,
                     delay=delay, seed=n + bits)
    nf = 37
    r1, r2 = random_raw(scan, nf, seed=n * 7 + bits)
    s = engine.open_scan(to_fxc(scan))
    x1, x2 = s.decode(dev(r1), dev(r2), nf, first_frame=3)
    s.check()
    x1, x2 = x1.cpu().numpy(), x2.cpu().numpy()
    ents = oracle.c_delay_entries(scan, 3, nf)
    bpf1, bpf2 = scan.bpf(bits), scan.bpf(bits)
    shifts = set()
    for i in range(nf):
        e1 = oracle.c_decode(r1[i * bpf1:(i + 1) * bpf1], n, bits, scan.shuffle1, scan.levels1, l1)
        e2 = oracle.c_decode(r2[i * bpf2:(i + 1) * bpf2], n, bits, scan.shuffle2, scan.levels2, l2)
        e1 = oracle.c_shift(e1, ents["int1"][i])
        e2 = oracle.c_shift(e2, ents["int2"][i])
        shifts.add(int(ents["int1"][i]))
        np.testing.assert_array_equal(x1[i], e1, err_msg=f"station 1 frame {i}")
        np.testing.assert_array_equal(x2[i], e2, err_msg=f"station 2 frame {i}")
    assert any(v > 0 for v in shifts) and any(v < 0 for v in shifts)
    assert any(abs(v) >= n for v in shifts)
    s.close()


def test_fft8192_decode_grid1_mixed_bits(engine):
    """The FFT-8192 kernel's decode with station 2 as its primary (grid 1),
    mixed bit depths and shuffle classes, LSB on station 2: bit-exact."""
    fs, n = 1024e6, 8192
    delay = dict(net_d1_base=-700 / fs, total_rate1_base=0.4, net_d2_base=3.0 / fs)
    scan = make_scan(fft=n, fs=fs, bits1=2, bits2=4, shuffle="generic", lsb2=True,
                     band=(-40, 40, 4096, 0), grid=1, delay=delay, seed=77)
    nf = 23
    r1, r2 = random_raw(scan, nf, seed=78)
    s = engine.open_scan(to_fxc(scan))
    x1, x2 = s.decode(dev(r1), dev(r2), nf, first_frame=1)
    s.check()
    x1, x2 = x1.cpu().numpy(), x2.cpu().numpy()
    ents = oracle.c_delay_entries(scan, 1, nf)
    b1, b2 = scan.bpf(2), scan.bpf(4)
    for i in range(nf):
        e1 = oracle.c_decode(r1[i * b1:(i + 1) * b1], n, 2, scan.shuffle1, scan.levels1, False)
        e2 = oracle.c_decode(r2[i * b2:(i + 1) * b2], n, 4, scan.shuffle2, scan.levels2, True)
        np.testing.assert_array_equal(x1[i], oracle.c_shift(e1, ents["int1"][i]))
        np.testing.assert_array_equal(x2[i], oracle.c_shift(e2, ents["int2"][i]))
    s.close()


@pytest.mark.parametrize("case", [c for c in KAT["decode"] if c["expect"] is not None
                                  and len(c["raw"]) == 4], ids=lambda c: c["name"])
def test_decode_kat_on_gpu(engine, case):
    """The hand-derived decode vectors, tiled to one 1024-sample frame."""
    bits = case["bits"]
    n = 1024
    per_word = 32 // bits
    reps = n // per_word
    raw = np.tile(np.array(case["raw"], np.uint8), reps)
    scan = make_scan(fft=n, bits1=bits, bits2=bits, levels1=case["levels"],
                     levels2=case["levels"])
    scan.shuffle1 = scan.shuffle2 = case["shuffle"]
    scan.lsb1 = scan.lsb2 = case["lsb"]
    s = engine.open_scan(to_fxc(scan))
    x1, x2 = s.decode(dev(raw), dev(raw), 1)
    s.check()
    exp = np.tile(np.array(case["expect"], np.float32), reps)
    np.testing.assert_array_equal(x1.cpu().numpy()[0], exp)
    np.testing.assert_array_equal(x2.cpu().numpy()[0], exp)


# ------------------------------------------------------------------- delay

@pytest.mark.parametrize("branch", ["table", "poly"])
def test_delay_model_bit_exact(engine, branch):
    fs = 1024e6
    n = 8192
    if branch == "table":
        table = 1e-7 + 3.1e-9 * np.arange(12) + 1e-12 * np.arange(12) ** 2
        delay = dict(coarse_delay_s=2.2e-8, delay_user_samples=0.3, extra_delay_rate_sps=1.3e-9,
                     clock1_delay_s=1e-7, clock1_rate_sps=1e-12, clock2_delay_s=2.5e-6,
                     clock2_rate_sps=-3e-12, d_seek=2.6e-6, lo1_hz=8.4e9, lo2_hz=8.2e9,
                     time_offset_s=3.0)
    else:
        table = None
        delay = dict(net_d1_base=-4.3e-7, total_rate1_base=3e-9, total_accel1_base=1e-10,
                     net_d2_base=1e-9, total_rate2_base=-2e-10, d_seek=1e-6, lo1_hz=6.7e9,
                     lo2_hz=6.7e9)
    scan = make_scan(fft=n, fs=fs, delay=delay, table=table)
    s = engine.open_scan(to_fxc(scan))
    first, nf = 123, 1250000 // 4
    got = s.delay_entries(first, nf)
    idx = np.r_[0:2000, nf - 2000:nf]
    ref = oracle.c_delay_entries(scan, first + int(idx[0]), 2000)
    ref2 = oracle.c_delay_entries(scan, first + nf - 2000, 2000)
    ref = np.concatenate([ref, ref2])
    g = got[idx]
    np.testing.assert_array_equal(g["int1"], ref["int1"])
    np.testing.assert_array_equal(g["int2"], ref["int2"])
    np.testing.assert_array_equal(g["frac1"], ref["frac1"])
    np.testing.assert_array_equal(g["frac2"], ref["frac2"])
    # f32 sin/cos of the same f32 angle: CUDA sincosf vs glibc, within 2 ulp
    np.testing.assert_allclose(g["fr_lo1"], ref["fr_lo1"], atol=2.5e-7)
    np.testing.assert_allclose(g["fr_lo2"], ref["fr_lo2"], atol=2.5e-7)
    s.close()


@pytest.mark.gpu
def test_delay_split_readme_examples(engine):
    """The reference's worked examples of the delay split (README.md:225-235):
    12.983 samples -> integer shift 13 and fraction -0.017 sample, 12.345 ->
    12 and +0.345, through the product's FP64 frame records on the GPU."""
    kat = json.loads((Path(__file__).parent / "golden" / "kat.json").read_text())
    for c in kat["readme"]["delay_split"]:
        fs = 1024e6
        scan = make_scan(fft=1024, fs=fs, delay=dict(net_d1_base=c["samples"] / fs))
        s = engine.open_scan(to_fxc(scan))
        e = s.delay_entries(0, 4)
        s.close()
        assert int(e["int1"][0]) == c["n"]
        assert abs(float(e["frac1"][0]) * fs - c["eps_samples"]) < 1e-9


# ----------------------------------------------------------------- spectra

@pytest.mark.parametrize("n", [1024, 2048, 4096, 8192])
def test_spectra_vs_fp64(engine, n):
    scan = make_scan(fft=n, fs=512e6, bits1=2, bits2=8, shuffle="generic", lsb1=True,
                     delay=DELAY)
    nf = 9
    r1, r2 = signal_raw(scan, nf, seed=n, rho=0.3, delay_samples=3.7)
    s = engine.open_scan(to_fxc(scan))
    s1, s2 = s.spectra(dev(r1), dev(r2), nf, first_frame=0)
    s.check()
    s1, s2 = s1.cpu().numpy(), s2.cpu().numpy()
    ents = oracle.np_delay_entries(scan, 0, nf)
    x1 = oracle.np_decode_frames(r1, nf, n, scan.bits1, scan.shuffle1, scan.levels1, True)
    x2 = oracle.np_decode_frames(r2, nf, n, scan.bits2, scan.shuffle2, scan.levels2, False)
    x1 = oracle.np_shift_frames(x1, np.array([e[0] for e in ents]))
    x2 = oracle.np_shift_frames(x2, np.array([e[1] for e in ents]))
    f1, f2 = np.fft.rfft(x1, axis=1), np.fft.rfft(x2, axis=1)
    for a, b, name in ((s1, f1, "S1"), (s2, f2, "S2")):
        err = np.abs(a - b).max() / np.sqrt(np.mean(np.abs(b) ** 2))
        assert err < 5e-6, (name, err)
    s.close()


# --------------------------------------------------------- sector products

SECTOR_CASES = [
    dict(fft=1024),
    dict(fft=1024, shuffle="generic", lsb1=True, band=(5, 0, 507, 5), grid=0),
    dict(fft=2048, shuffle="pairswap", lsb2=True, band=(-7, 7, 1024, 0), grid=1),
    dict(fft=4096, bits1=4, bits2=4, shuffle="generic", band=(40, 0, 2008, 40), grid=1),
    dict(fft=8192, shuffle="generic", lsb1=True, band=(128, 0, 3968, 128), grid=0),
    dict(fft=8192, bits1=1, bits2=8, band=(-128, 128, 4096, 0), grid=0),
    dict(fft=1024, products=oracle.PROD_ACF | oracle.PROD_ACF_OVERLAP_ONLY, band=(3, 0, 509, 3)),
    dict(fft=2048, products=oracle.PROD_XCF, band=(0, 0, 1024, 0)),
    dict(fft=4096, products=oracle.PROD_ACF | oracle.PROD_ACF_OVERLAP_ONLY,
         band=(-9, 9, 2048, 0), grid=1),
    # FFT 8192 (its own kernel): every decode variant, both grids, LSB on
    # either station, product subsets
    dict(fft=8192, shuffle="pairswap", lsb2=True, band=(-40, 40, 4096, 0), grid=1),
    dict(fft=8192, bits1=4, bits2=2, shuffle="generic", lsb1=True, lsb2=True,
         band=(64, 0, 4032, 64), grid=1),
    dict(fft=8192, bits1=8, bits2=4, shuffle="generic", band=(0, 0, 4096, 0),
         products=oracle.PROD_ACF | oracle.PROD_ACF_OVERLAP_ONLY | oracle.PROD_XCF),
    dict(fft=8192, shuffle="sample2", lsb1=True, band=(16, 0, 4080, 16), grid=1,
         products=oracle.PROD_XCF),
    dict(fft=8192, bits1=1, bits2=1, shuffle="generic", lsb2=True, band=(-3, 3, 4096, 0),
         products=oracle.PROD_ACF),
]


@pytest.mark.parametrize("kw", SECTOR_CASES)
@pytest.mark.parametrize("nf", [1, 7, 301])
def test_sector_vs_fp64(engine, kw, nf):
    scan = make_scan(delay=DELAY, fs=512e6, **kw)
    r1, r2 = signal_raw(scan, nf, seed=nf + kw.get("fft", 0), rho=0.2, delay_samples=6.4)
    s = engine.open_scan(to_fxc(scan))
    got = s.sector_device(dev(r1), dev(r2), nf, first_frame=11)
    ref = oracle.fp64_sector_corr(scan, r1, r2, nf, first_frame=11)
    ref_acf = ref
    if not scan.products & oracle.PROD_ACF or scan.products & oracle.PROD_ACF_OVERLAP_ONLY:
        full = dataclasses.replace(scan, products=oracle.PROD_ACF)
        ref_acf = oracle.fp64_sector_corr(full, r1, r2, nf, first_frame=11)
    assert_sector_close(got, ref, scan, f"gpu vs fp64 {kw} nf={nf}", nf=nf, ref_acf=ref_acf)
    # the f32 restatement of the reference agrees within its own drift
    c = oracle.c_sector_corr(scan, r1, r2, nf, first_frame=11)
    for k in ("acf11", "acf22"):
        if scan.products & oracle.PROD_ACF:
            rel, ph, ab = spectral_errors(got[k], c[k])
            assert rel < 1e-5, (k, rel)
    if scan.products & oracle.PROD_XCF:
        # the restatement keeps the reference's f32 phase-ramp recurrence: its
        # own drift from FP64 stays inside the recurrence bound, and the GPU
        # sits within that drift plus the GPU's FP64 tolerance of it
        fl = xcf_floor(ref_acf, nf)
        _, a1s, a1e, _ = scan.band_or_default()
        bound = xcf_drift_bound(a1e - a1s)
        rel_c, ph_c, _ = spectral_errors(c["xcf"], ref["xcf"], fl)
        assert rel_c <= bound["rel_amp"] and ph_c <= bound["phase_rad"], (rel_c, ph_c, bound)
        rel, ph, ab = spectral_errors(got["xcf"], c["xcf"], fl)
        assert rel <= 1.01 * rel_c + REL_AMP_TOL and ph <= 1.01 * ph_c + PHASE_TOL, (
            rel, ph, rel_c, ph_c)
    # products not requested are exactly zero
    if not scan.products & oracle.PROD_XCF:
        assert np.all(got["xcf"] == 0)
    if not scan.products & oracle.PROD_ACF:
        assert np.all(got["acf11"] == 0) and np.all(got["acf22"] == 0)
    s.close()


@pytest.mark.parametrize("fft,nf", [(1024, 20000), (4096, 6000), (8192, 3000), (16384, 600)])
def test_weak_correlation_long_integration(engine, fft, nf):
    """rho = 0.01 over thousands of frames: the shared complex FFT's
    cross-station rounding leak must not accumulate into the cross-spectrum
    (it would reach ~1e-6 * sqrt(nf) of the XCF noise floor)."""
    scan = make_scan(fft=fft, fs=512e6, delay=DELAY, shuffle="generic", lsb1=True,
                     band=(8, 0, fft // 2 - 8, 8))
    r1, r2 = signal_raw(scan, nf, seed=fft + 1, rho=0.01, delay_samples=3.3)
    s = engine.open_scan(to_fxc(scan))
    got = s.sector_device(dev(r1), dev(r2), nf, first_frame=5)
    ref = oracle.fp64_sector_corr(scan, r1, r2, nf, first_frame=5)
    assert_sector_close(got, ref, scan, f"rho=0.01 fft={fft} nf={nf}", nf=nf, ref_acf=ref)
    s.close()


@pytest.mark.parametrize("fft,d1,sb", [
    (8192, -2.3e-6, 128), (8192, 5.1e-6, 128), (8192, 1.7e-5, 128),
    (16384, -9.1e-6, 128), (16384, 2.0e-6, 128), (16384, 3.3e-5, 128),
    # the cluster kernel: staged column ranges clamped at either end of the
    # frame, whole ranges outside it, and (odd sb) secondary spectra exchanged
    # between the CTAs of a cluster
    (16384, -9.1e-6, 129), (32768, -9.1e-6, 128), (32768, 3.3e-5, 131), (32768, 7.0e-5, 128),
    (65536, -5.3e-5, 133), (65536, 2.0e-6, 128), (65536, 1.4e-4, 128)])
def test_sector_large_shift(engine, fft, d1, sb):
    """Integer shifts beyond N/16 (and beyond N: an all-zero station frame)."""
    delay = dict(DELAY, net_d1_base=d1)
    scan = make_scan(fft=fft, fs=512e6, delay=delay, shuffle="generic", lsb1=True,
                     band=(sb, 0, fft // 2 - sb, sb))
    nf = 9
    r1, r2 = signal_raw(scan, nf, seed=5, rho=0.2, delay_samples=6.4)
    s = engine.open_scan(to_fxc(scan))
    got = s.sector_device(dev(r1), dev(r2), nf, first_frame=3)
    ref = oracle.fp64_sector_corr(scan, r1, r2, nf, first_frame=3)
    if not np.any(ref["acf11"]):  # shift >= N: station 1 frames are all zero
        # only rounding leakage of the shared complex FFT remains
        scale = float(ref["acf22"].max())
        assert float(np.abs(got["acf11"]).max()) < 1e-10 * scale
        assert float(np.abs(got["xcf"]).max()) < 1e-6 * scale
        rel, ph, ab = spectral_errors(got["acf22"], ref["acf22"])
        assert rel < 1e-5, rel
    else:
        assert_sector_close(got, ref, scan, f"large shift {d1}", nf=nf, ref_acf=ref)
    s.close()


def test_sector_empty_and_deterministic(engine):
    scan = make_scan(fft=4096, fs=512e6, delay=DELAY, band=(40, 0, 2008, 40))
    s = engine.open_scan(to_fxc(scan))
    nf = 1000
    r1, r2 = signal_raw(scan, nf, seed=4, rho=0.1)
    d1, d2 = dev(r1), dev(r2)
    a = s.sector_device(d1, d2, nf)
    b = s.sector_device(d1, d2, nf)
    for k in ("acf11", "acf22", "xcf"):
        assert np.array_equal(a[k], b[k]), k  # fixed-order reduction
    z = s.sector_device(d1, d2, 0)
    assert all(np.all(z[k] == 0) for k in ("acf11", "acf22", "xcf"))
    s.close()


def test_sector_additivity(engine):
    """Splitting a sector into pieces (with the right first_frame) sums to
    the whole: a size-independent property used at full size in the bench
    config tests."""
    scan = make_scan(fft=8192, fs=1024e6, delay=DELAY, band=(128, 0, 3968, 128),
                     shuffle="generic", lsb1=True)
    s = engine.open_scan(to_fxc(scan))
    nf = 2000
    r1, r2 = random_raw(scan, nf, seed=9)
    whole = s.sector_device(dev(r1), dev(r2), nf, first_frame=50)
    b = scan.bpf(2)
    p1 = s.sector_device(dev(r1[:700 * b]), dev(r2[:700 * b]), 700, first_frame=50)
    p2 = s.sector_device(dev(r1[700 * b:]), dev(r2[700 * b:]), 1300, first_frame=750)
    for k in ("acf11", "acf22", "xcf"):
        assert_spectra_close(p1[k] + p2[k], whole[k], k)
    s.close()


def test_host_submit_wait_matches_device_path(engine):
    scan = make_scan(fft=8192, fs=1024e6, delay=DELAY, band=(128, 0, 3968, 128),
                     shuffle="generic", lsb1=True)
    s = engine.open_scan(to_fxc(scan))
    nf = 500
    sectors = [signal_raw(scan, nf, seed=30 + i, rho=0.1) for i in range(4)]
    ids = []
    results = []
    for i, (r1, r2) in enumerate(sectors):
        if len(ids) == 3:
            results.append(s.wait(ids.pop(0)))
        ids.append(s.submit(r1, r2, nf, first_frame=i * nf))
    while ids:
        results.append(s.wait(ids.pop(0)))
    for i, (r1, r2) in enumerate(sectors):
        ref = s.sector_device(dev(r1), dev(r2), nf, first_frame=i * nf)
        for k in ("acf11", "acf22", "xcf"):
            assert np.array_equal(results[i][k], ref[k]), (i, k)
    with pytest.raises(Exception):
        s.wait(12345)
    s.close()


def test_parseval_full_sector(engine):
    """Full-size check (1024 Msps, N=8192, one 1-s sector of 125000 frames)
    through a size-independent identity: with no shift, the one-sided ACF
    satisfies |X0|^2 + |X_N/2|^2 + 2 sum_k |X_k|^2 = N sum_n x[n]^2 per frame,
    checked exactly on a 1000-frame chunk against the decoded samples, and
    statistically over the whole sector (E[x^2] = 5 for uniform codes)."""
    import torch

    n, nf = 8192, 125000
    scan = make_scan(fft=n, fs=1024e6, levels1=[-3.0, -1.0, 1.0, 3.0],
                     levels2=[-3.0, -1.0, 1.0, 3.0], shuffle="generic", lsb1=True)
    s = engine.open_scan(to_fxc(scan))
    g = torch.Generator(device="cuda").manual_seed(5)
    r1 = torch.randint(0, 256, (nf * 2048,), dtype=torch.uint8, device="cuda", generator=g)
    r2 = torch.randint(0, 256, (nf * 2048,), dtype=torch.uint8, device="cuda", generator=g)
    res = s.sector_device(r1, r2, nf)

    acc = res["acf11"]
    one_sided = acc[0] + acc[-1] + 2 * acc[1:-1].sum()
    x1, _ = s.decode(r1[: 1000 * 2048], r2[: 1000 * 2048], 1000)
    e_chunk = float((x1.double() ** 2).sum())
    res_chunk = s.sector_device(r1[: 1000 * 2048], r2[: 1000 * 2048], 1000)
    a = res_chunk["acf11"]
    assert math.isclose(a[0] + a[-1] + 2 * a[1:-1].sum(), n * e_chunk, rel_tol=2e-6)
    # whole sector: E[x^2] = 5 for uniform codes over {+-1, +-3}; 1e9 samples
    assert math.isclose(one_sided / (n * nf * n), 5.0, rel_tol=2e-3)
    s.close()


# ------------------------------------------------- FFT lengths above 8192

@pytest.mark.parametrize("n", [16384, 32768, 65536])
def test_large_decode_bit_exact(engine, n):
    fs = 512e6
    delay = dict(net_d1_base=-0.6 * n / fs, total_rate1_base=0.05, net_d2_base=7.0 / fs)
    scan = make_scan(fft=n, fs=fs, bits1=2, bits2=4, shuffle="generic", lsb1=True, delay=delay,
                     seed=n)
    nf = 5
    r1, r2 = random_raw(scan, nf, seed=n + 1)
    s = engine.open_scan(to_fxc(scan))
    x1, x2 = s.decode(dev(r1), dev(r2), nf, first_frame=2)
    s.check()
    x1, x2 = x1.cpu().numpy(), x2.cpu().numpy()
    ents = oracle.c_delay_entries(scan, 2, nf)
    b1, b2 = scan.bpf(2), scan.bpf(4)
    for i in range(nf):
        e1 = oracle.c_decode(r1[i * b1:(i + 1) * b1], n, 2, scan.shuffle1, scan.levels1, True)
        e2 = oracle.c_decode(r2[i * b2:(i + 1) * b2], n, 4, scan.shuffle2, scan.levels2, False)
        np.testing.assert_array_equal(x1[i], oracle.c_shift(e1, ents["int1"][i]))
        np.testing.assert_array_equal(x2[i], oracle.c_shift(e2, ents["int2"][i]))
    s.close()


@pytest.mark.parametrize("n", [16384, 65536])
def test_large_spectra_vs_fp64(engine, n):
    scan = make_scan(fft=n, fs=512e6, bits1=2, bits2=8, shuffle="generic", lsb1=True,
                     delay=DELAY)
    nf = 3
    r1, r2 = signal_raw(scan, nf, seed=n, rho=0.3, delay_samples=3.7)
    s = engine.open_scan(to_fxc(scan))
    s1, s2 = s.spectra(dev(r1), dev(r2), nf, first_frame=0)
    s.check()
    s1, s2 = s1.cpu().numpy(), s2.cpu().numpy()
    ents = oracle.np_delay_entries(scan, 0, nf)
    x1 = oracle.np_decode_frames(r1, nf, n, scan.bits1, scan.shuffle1, scan.levels1, True)
    x2 = oracle.np_decode_frames(r2, nf, n, scan.bits2, scan.shuffle2, scan.levels2, False)
    x1 = oracle.np_shift_frames(x1, np.array([e[0] for e in ents]))
    x2 = oracle.np_shift_frames(x2, np.array([e[1] for e in ents]))
    f1, f2 = np.fft.rfft(x1, axis=1), np.fft.rfft(x2, axis=1)
    for a, b, name in ((s1, f1, "S1"), (s2, f2, "S2")):
        err = np.abs(a - b).max() / np.sqrt(np.mean(np.abs(b) ** 2))
        assert err < 5e-6, (name, err)
    s.close()


LARGE_CASES = [
    dict(fft=16384, band=(256, 0, 7936, 256), grid=0, shuffle="generic", lsb1=True),
    # FFT 16384, two-row kernel: grid 1, LSB on station 2, pair-splitting 2-bit and 4-bit
    dict(fft=16384, band=(-40, 40, 8192, 0), grid=1, shuffle="generic", lsb2=True),
    dict(fft=16384, bits1=4, bits2=2, band=(12, 0, 8180, 12), grid=0, shuffle="pairswap",
         products=oracle.PROD_ACF | oracle.PROD_ACF_OVERLAP_ONLY | oracle.PROD_XCF),
    # odd band shift, 1- and 2-bit stations: both rows in one CTA, each row's
    # secondary spectra in the other row's slots
    dict(fft=16384, band=(-7, 7, 8192, 0), grid=0, lsb1=True),
    dict(fft=16384, band=(5, 0, 8187, 5), grid=1, bits1=1, bits2=2, shuffle="pairswap", lsb2=True,
         products=oracle.PROD_ACF | oracle.PROD_ACF_OVERLAP_ONLY | oracle.PROD_XCF),
    # odd band shift, 8-bit stations: the cluster kernel, secondary spectra
    # exchanged between CTAs
    dict(fft=16384, band=(3, 0, 8190, 3), grid=1, bits1=8, bits2=8, shuffle="generic"),
    dict(fft=32768, band=(-6, 6, 16385, 0), grid=0, bits1=2, bits2=1, shuffle="sample2",
         lsb2=True),
    dict(fft=65536, band=(13, 0, 32755, 13), grid=1, shuffle="generic", lsb1=True),
    dict(fft=32768, band=(-64, 64, 16384, 0), grid=1, bits1=4, bits2=4),
    dict(fft=65536, band=(0, 0, 32768, 0), grid=0, bits1=1, bits2=2,
         products=oracle.PROD_ACF | oracle.PROD_ACF_OVERLAP_ONLY | oracle.PROD_XCF),
    # shuffled 1- and 2-bit stations (bits kept together, reordered, split or
    # swapped), and the generic 8/4-bit path
    dict(fft=32768, band=(64, 0, 16320, 64), grid=0, shuffle="generic", lsb2=True),
    dict(fft=32768, band=(0, 0, 16384, 0), grid=1, bits1=1, bits2=2, shuffle="pairswap",
         lsb1=True),
    dict(fft=16384, band=(5, 0, 8187, 5), grid=1, shuffle="sample2"),
    dict(fft=65536, band=(-32, 32, 32768, 0), grid=0, bits1=8, bits2=4, shuffle="generic"),
]


@pytest.mark.parametrize("kw", LARGE_CASES)
@pytest.mark.parametrize("nf", [1, 37])
def test_large_sector_vs_fp64(engine, kw, nf):
    scan = make_scan(delay=DELAY, fs=512e6, **kw)
    r1, r2 = signal_raw(scan, nf, seed=nf + kw["fft"], rho=0.2, delay_samples=6.4)
    s = engine.open_scan(to_fxc(scan))
    got = s.sector_device(dev(r1), dev(r2), nf, first_frame=3)
    ref = oracle.fp64_sector_corr(scan, r1, r2, nf, first_frame=3)
    assert_sector_close(got, ref, scan, f"gpu vs fp64 {kw} nf={nf}", nf=nf)
    s.close()


def test_host_register_submit(engine, fxc_lib):
    """Caller-owned sector buffers page-locked in place (fxc_host_register)
    give the same results through fxc_sector_submit/wait as pageable ones."""
    scan = make_scan(fft=8192, fs=1024e6, delay=DELAY, band=(128, 0, 3968, 128),
                     shuffle="generic", lsb1=True)
    nf = 400
    r1, r2 = signal_raw(scan, nf, seed=41, rho=0.1)
    s = engine.open_scan(to_fxc(scan))
    plain = s.wait(s.submit(r1, r2, nf, first_frame=8))
    b1, b2 = np.array(r1), np.array(r2)
    fxc_lib.host_register(b1)
    fxc_lib.host_register(b2)
    fxc_lib.host_register(b2)  # already registered: accepted
    try:
        pinned = s.wait(s.submit(b1, b2, nf, first_frame=8))
    finally:
        fxc_lib.host_unregister(b1)
        fxc_lib.host_unregister(b2)
    for k in ("acf11", "acf22", "xcf"):
        assert np.array_equal(plain[k], pinned[k]), k
    with pytest.raises(fxc_lib.FxcError):
        fxc_lib.host_unregister(b1)  # no longer registered
    s.close()
