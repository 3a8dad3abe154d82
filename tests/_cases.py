"""Shared test cases: scan builders, seeded inputs and the spectral
comparison used by every parity test.

Tolerance (stated against the FP64 oracle, as the correlation path is
floating point): per-bin relative amplitude error <= 1e-5 and phase error
<= 1e-4 rad.  A bin's relative error is taken against max(|ref|, floor):
for auto-spectra floor = 5% of the product's RMS; for a cross-spectrum bin
floor = sqrt(<acf11>*<acf22>/nf) with <.> a 33-bin running mean, the
expected amplitude of a noise-only bin after nf frames, because f32 rounding
errors of a cross-spectrum scale with that noise amplitude and not with the
(possibly near-zero) realised value.
Phase errors are checked on bins at or above the floor.  On all bins the
absolute error must also stay <= 1e-5 * RMS of the product.
"""
from __future__ import annotations

import dataclasses

import numpy as np

import oracle

REL_AMP_TOL = 1e-5
PHASE_TOL = 1e-4
FLOOR = 0.05


def make_scan(fft=1024, fs=32e6, bits1=2, bits2=2, shuffle="identity", lsb1=False, lsb2=False,
              band=None, grid=0, products=oracle.PROD_ACF | oracle.PROD_XCF, delay=None,
              table=None, levels1=None, levels2=None, seed=0, w1=1.0, w2=1.0):
    def sh(kind, s):
        if kind == "identity":
            return list(range(32))
        if kind == "pairswap":
            return [i ^ 1 for i in range(32)]
        if kind == "sample2":  # whole 2-bit samples reordered, bits kept in order
            order = np.random.Generator(np.random.PCG64(s)).permutation(16)
            return [2 * int(order[i >> 1]) + (i & 1) for i in range(32)]
        return oracle.random_shuffle(s)

    return oracle.Scan(
        fft=fft, fs=fs, bits1=bits1, bits2=bits2,
        levels1=levels1 or oracle.default_levels(bits1),
        levels2=levels2 or oracle.default_levels(bits2),
        shuffle1=sh(shuffle, seed + 11), shuffle2=sh(shuffle, seed + 12),
        lsb1=lsb1, lsb2=lsb2, band=band, grid=grid, products=products, w1=w1, w2=w2,
        delay=dict(delay or {}), geom_table=None if table is None else np.asarray(table, float))


def to_fxc(scan: oracle.Scan):
    import fxc

    d = dataclasses.asdict(scan)
    d["geom_table"] = scan.geom_table
    return fxc.ScanConfig(**d)


def random_raw(scan, nf, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    r1 = rng.integers(0, 256, nf * scan.bpf(scan.bits1), dtype=np.uint8)
    r2 = rng.integers(0, 256, nf * scan.bpf(scan.bits2), dtype=np.uint8)
    return r1, r2


def signal_raw(scan, nf, seed, rho=0.05, delay_samples=0.0, tone_bin=None):
    """Seeded quantised Gaussian streams with a common component (rho) whose
    copy at station 2 is delayed by delay_samples."""
    n = nf * scan.fft
    x1, x2 = oracle.synth_station_pair(n, seed, rho=rho, delay_samples=delay_samples,
                                       tone_bin=tone_bin, fft=scan.fft)
    r1 = oracle.encode_station(x1, scan.bits1, scan.levels1, scan.shuffle1, scan.lsb1)
    r2 = oracle.encode_station(x2, scan.bits2, scan.levels2, scan.shuffle2, scan.lsb2)
    return r1, r2


def spectral_errors(a, b, floor=None):
    """(max relative amplitude error, max phase error, max complex error /
    peak |b|) of a against reference b; `floor` (scalar or per bin) bounds the
    relative-error denominator from below (default 5% of rms(|b|))."""
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    mag = np.abs(b)
    rms = float(np.sqrt(np.mean(mag ** 2))) if mag.size else 0.0
    if rms == 0.0:
        return 0.0, 0.0, float(np.abs(a).max()) if a.size else 0.0
    fl = FLOOR * rms if floor is None else np.maximum(np.asarray(floor, float), 1e-300)
    fl = np.broadcast_to(fl, mag.shape)
    den = np.maximum(mag, fl)
    rel = float(np.max(np.abs(np.abs(a) - mag) / den))
    m = (mag >= fl) & (mag > 0)
    ph = float(np.max(np.abs(np.angle(a[m] * np.conj(b[m]))))) if m.any() else 0.0
    ab = float(np.max(np.abs(a - b)) / np.max(mag))
    return rel, ph, ab


def assert_spectra_close(a, b, what, rel_tol=REL_AMP_TOL, phase_tol=PHASE_TOL, floor=None):
    rel, ph, ab = spectral_errors(a, b, floor)
    assert rel <= rel_tol and ph <= phase_tol and ab <= rel_tol, (
        f"{what}: rel amp {rel:.3e} (tol {rel_tol}), phase {ph:.3e} rad (tol {phase_tol}), "
        f"abs/peak {ab:.3e}")
    return rel, ph, ab


def _running_mean(x, w=33):
    k = np.ones(w)
    num = np.convolve(x, k, mode="same")
    den = np.convolve(np.ones_like(x), k, mode="same")
    return num / den


def xcf_floor(ref, nf):
    """Expected noise amplitude sqrt(<acf11><acf22>/nf) of each cross-spectrum
    bin (33-bin running means of the auto-spectra), or None when the reference
    has no auto-spectra."""
    a11, a22 = np.asarray(ref["acf11"]), np.asarray(ref["acf22"])
    if not (np.any(a11) and np.any(a22)) or nf <= 0:
        return None
    return np.sqrt(np.maximum(_running_mean(a11) * _running_mean(a22), 0.0) / nf)


def assert_sector_close(got, ref, scan, what, nf=None, ref_acf=None):
    """ref_acf: a reference holding both auto-spectra on the grid (defaults
    to ref) for the cross-spectrum floor."""
    out = {}
    if scan.products & oracle.PROD_ACF:
        out["acf11"] = assert_spectra_close(got["acf11"], ref["acf11"], what + " acf11")
        out["acf22"] = assert_spectra_close(got["acf22"], ref["acf22"], what + " acf22")
    if scan.products & oracle.PROD_XCF:
        fl = xcf_floor(ref_acf if ref_acf is not None else ref, nf) if nf else None
        out["xcf"] = assert_spectra_close(got["xcf"], ref["xcf"], what + " xcf", floor=fl)
    return out


def xcf_drift_bound(ov):
    """How far the reference's XCF may sit from the exact product: its phase
    ramp is the f32 recurrence ph *= step over the ov overlap bins
    (src/main.rs:2513-2527, src/utils.rs:115-117), so after k bins the ramp's
    relative magnitude and its angle each carry up to k roundings of about
    2^-24, plus the rounding of step itself: at most ov * 2^-23 in both.  The
    GPU evaluates the ramp per bin and tracks FP64 within REL_AMP_TOL /
    PHASE_TOL, so the GPU against the f32 restatement is bounded by the sum."""
    d = ov * 2.0 ** -23
    return {"rel_amp": REL_AMP_TOL + d, "phase_rad": PHASE_TOL + d}
