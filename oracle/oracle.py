"""CPU oracle for the fx-corr correlation path.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` import this
module, and only as the checker or as the timed CPU baseline.  The product
(``libfxc.so``, the CLI) never imports, links or calls anything here.

Two oracles live here:

* ``C`` — a ctypes binding of ``fxc_oracle.c``, a line-cited f32/f64
  restatement of the reference's rayon CPU path (same types, same operation
  order where the reference fixes it; the FFT is a project-written Stockham
  FFT because rustfft/realfft sources are not available).
* ``fp64_*`` — a NumPy float64 restatement of the same path: same decode and
  the same f64 delay model (so the same integer shifts), but float64 FFTs,
  float64 fringe phasors and an exact per-bin phase ramp.  This is the
  mathematical truth that precision claims are stated against.

Parity status: UNPINNED by reference-produced vectors (the Rust reference
cannot be built in this environment and ships no fixtures for this path);
pinned by hand-derived known-answer vectors in tests/golden.

Reference citations are relative to the fx-corr project root.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_DIR = HERE / "lib"
LIB_PATH = LIB_DIR / "libfxc_oracle.so"

PROD_ACF, PROD_XCF, PROD_PHASED, PROD_RAW, PROD_ACF_OVERLAP_ONLY = 1, 2, 4, 8, 16

# args.rs:9-12 — DEFAULT_SHUFFLE_IN (external, MSB first) -> identity internally
DEFAULT_SHUFFLE_EXT = list(range(31, -1, -1))


def build(force: bool = False) -> Path:
    """Compile the C restatement into oracle/lib/libfxc_oracle.so."""
    srcs = [HERE / "fxc_oracle.c", HERE / "synth.c"]
    if LIB_PATH.exists() and not force and LIB_PATH.stat().st_mtime >= max(
        [x.stat().st_mtime for x in srcs] + [(HERE / "fxc_oracle.h").stat().st_mtime]
    ):
        return LIB_PATH
    LIB_DIR.mkdir(exist_ok=True)
    tmp = LIB_PATH.with_suffix(f".so.tmp{os.getpid()}")
    cmd = [
        "gcc", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-math-errno",
        "-fopenmp", "-fPIC", "-shared", "-std=c11", "-D_GNU_SOURCE",
        "-o", str(tmp), *map(str, srcs), "-lm",
    ]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


# ----------------------------------------------------------------- ctypes

class DelayCfg(C.Structure):
    """DelayEvalConfig (src/main.rs:161-182)."""

    _fields_ = [
        ("frame_dt", C.c_double), ("fs", C.c_double), ("time_offset_s", C.c_double),
        ("geom_table", C.POINTER(C.c_double)), ("geom_len", C.c_uint64),
        ("coarse_delay_s", C.c_double), ("delay_user_samples", C.c_double),
        ("extra_delay_rate_sps", C.c_double),
        ("clock1_delay_s", C.c_double), ("clock1_rate_sps", C.c_double),
        ("clock2_delay_s", C.c_double), ("clock2_rate_sps", C.c_double),
        ("d_seek", C.c_double),
        ("net_d1_base", C.c_double), ("total_rate1_base", C.c_double),
        ("total_accel1_base", C.c_double),
        ("net_d2_base", C.c_double), ("total_rate2_base", C.c_double),
        ("total_accel2_base", C.c_double),
        ("lo1_hz", C.c_double), ("lo2_hz", C.c_double),
    ]


class FrameDelay(C.Structure):
    _fields_ = [
        ("int1", C.c_int64), ("int2", C.c_int64), ("frac1", C.c_double),
        ("frac2", C.c_double), ("fr_lo1", C.c_float * 2), ("fr_lo2", C.c_float * 2),
    ]


class ScanCfg(C.Structure):
    _fields_ = [
        ("fft_len", C.c_uint32), ("bits1", C.c_uint32), ("bits2", C.c_uint32),
        ("bits_out", C.c_uint32), ("fs_hz", C.c_double),
        ("levels1", C.c_double * 256), ("levels2", C.c_double * 256),
        ("nlevels1", C.c_uint32), ("nlevels2", C.c_uint32),
        ("shuffle1", C.c_uint8 * 32), ("shuffle2", C.c_uint8 * 32),
        ("lsb1", C.c_int32), ("lsb2", C.c_int32), ("shift_bins", C.c_int32),
        ("a1s", C.c_uint32), ("a1e", C.c_uint32), ("a2s", C.c_uint32),
        ("grid", C.c_int32), ("products", C.c_uint32),
        ("w1", C.c_double), ("w2", C.c_double), ("delay", DelayCfg),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        u8p, f32p, f64p = C.POINTER(C.c_uint8), C.POINTER(C.c_float), C.POINTER(C.c_double)
        L.orc_parse_shuffle.argtypes = [C.POINTER(C.c_int32), u8p]
        L.orc_decode.argtypes = [u8p, C.c_uint64, C.c_uint64, C.c_uint32, u8p, f64p, C.c_uint32,
                                 C.c_int32, f32p]
        L.orc_decode.restype = C.c_int64
        L.orc_shift_zerofill.argtypes = [f32p, C.c_uint64, C.c_int64]
        L.orc_rfft_f32.argtypes = [C.c_uint32, f32p, f32p]
        L.orc_irfft_f32.argtypes = [C.c_uint32, f32p, f32p]
        L.orc_delay_entry.argtypes = [C.POINTER(DelayCfg), C.c_uint64, C.POINTER(FrameDelay)]
        L.orc_band_alignment.argtypes = [C.c_uint32, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.POINTER(C.c_int64)]
        L.orc_xcf_phase_start_and_step.argtypes = [C.c_double, C.c_double, C.c_double,
                                                   C.c_uint64, C.c_uint64, f32p]
        L.orc_quantise_frame.argtypes = [f32p, C.c_uint64, C.c_uint32, f64p, C.c_uint32, u8p,
                                         u8p, C.c_uint64]
        L.orc_quantise_frame.restype = C.c_int64
        L.orc_sector_corr.argtypes = [C.POINTER(ScanCfg), u8p, u8p, C.c_uint64, C.c_uint64,
                                      f64p, f64p, f64p, C.c_int32]
        L.orc_sector_corr.restype = C.c_int64
        L.orc_sector_phased.argtypes = [C.POINTER(ScanCfg), u8p, u8p, C.c_uint64, C.c_uint64,
                                        f64p, u8p, C.c_int32]
        L.orc_sector_phased.restype = C.c_int64
        L.orc_normalize.argtypes = [C.c_uint32, C.c_uint64, C.c_double, f64p, f64p, f32p]
        L.orc_level_power.argtypes = [f64p, C.c_uint32]
        L.orc_level_power.restype = C.c_double
        L.orc_synth_pack_pair.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_uint32,
                                          C.c_double, C.c_double, C.c_double,
                                          C.c_uint32, f64p, C.c_uint32, C.c_double, u8p,
                                          C.c_int32, u8p, C.c_int32, u8p, u8p, C.c_int32]
        L.orc_synth_pack_pair.restype = C.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


# ------------------------------------------------------------- scan model

@dataclass
class Scan:
    """Everything one scan's hot path needs (the fields of the C-ABI's scan
    config).  Defaults follow the reference's CLI defaults (args.rs)."""

    fft: int = 1024
    fs: float = 32e6
    bits1: int = 2
    bits2: int = 2
    levels1: list = field(default_factory=lambda: [-1.5, -0.5, 0.5, 1.5])
    levels2: list = field(default_factory=lambda: [-1.5, -0.5, 0.5, 1.5])
    shuffle1: list = field(default_factory=lambda: list(range(32)))  # internal map
    shuffle2: list = field(default_factory=lambda: list(range(32)))
    lsb1: bool = False
    lsb2: bool = False
    band: tuple = None  # (sb, a1s, a1e, a2s); None -> full band, no shift
    grid: int = 0
    products: int = PROD_ACF | PROD_XCF
    w1: float = 1.0
    w2: float = 1.0
    delay: dict = field(default_factory=dict)  # DelayEvalConfig fields
    geom_table: np.ndarray = None

    @property
    def h(self):
        return self.fft // 2 + 1

    @property
    def bits_out(self):
        return max(self.bits1, self.bits2)

    def bpf(self, bits):
        return (self.fft * bits + 7) // 8

    def band_or_default(self):
        if self.band is not None:
            return self.band
        return (0, 0, self.fft // 2, 0)

    def delay_cfg_dict(self):
        d = dict(frame_dt=self.fft / self.fs, fs=self.fs, time_offset_s=0.0,
                 coarse_delay_s=0.0, delay_user_samples=0.0, extra_delay_rate_sps=0.0,
                 clock1_delay_s=0.0, clock1_rate_sps=0.0, clock2_delay_s=0.0,
                 clock2_rate_sps=0.0, d_seek=0.0, net_d1_base=0.0, total_rate1_base=0.0,
                 total_accel1_base=0.0, net_d2_base=0.0, total_rate2_base=0.0,
                 total_accel2_base=0.0, lo1_hz=0.0, lo2_hz=0.0)
        d.update(self.delay)
        return d

    def to_c(self) -> ScanCfg:
        c = ScanCfg()
        c.fft_len, c.bits1, c.bits2, c.bits_out = self.fft, self.bits1, self.bits2, self.bits_out
        c.fs_hz = self.fs
        for i, v in enumerate(self.levels1):
            c.levels1[i] = v
        for i, v in enumerate(self.levels2):
            c.levels2[i] = v
        c.nlevels1, c.nlevels2 = len(self.levels1), len(self.levels2)
        for i in range(32):
            c.shuffle1[i], c.shuffle2[i] = self.shuffle1[i], self.shuffle2[i]
        c.lsb1, c.lsb2 = int(self.lsb1), int(self.lsb2)
        sb, a1s, a1e, a2s = self.band_or_default()
        c.shift_bins, c.a1s, c.a1e, c.a2s = sb, a1s, a1e, a2s
        c.grid, c.products, c.w1, c.w2 = self.grid, self.products, self.w1, self.w2
        for k, v in self.delay_cfg_dict().items():
            setattr(c.delay, k, v)
        if self.geom_table is not None:
            self._gt = np.ascontiguousarray(self.geom_table, dtype=np.float64)
            c.delay.geom_table = _p(self._gt, C.c_double)
            c.delay.geom_len = len(self._gt)
        return c


# ------------------------------------------------------ C oracle wrappers

def parse_shuffle(ext) -> list:
    e = (C.c_int32 * 32)(*ext)
    out = (C.c_uint8 * 32)()
    if lib().orc_parse_shuffle(e, out) != 0:
        raise ValueError("Shuffle map must be a permutation of 0..31")
    return list(out)


def c_decode(raw: np.ndarray, samples: int, bits: int, shuffle, levels, lsb: bool):
    raw = np.ascontiguousarray(raw, dtype=np.uint8)
    out = np.zeros(max(samples, 1), np.float32)
    sh = np.asarray(shuffle, np.uint8)
    lv = np.asarray(levels, np.float64)
    r = lib().orc_decode(_p(raw, C.c_uint8), raw.size, samples, bits, _p(sh, C.c_uint8),
                         _p(lv, C.c_double), lv.size, int(lsb), _p(out, C.c_float))
    if r < 0:
        return None
    return out[:samples]


def c_shift(x: np.ndarray, s: int) -> np.ndarray:
    y = np.ascontiguousarray(x, dtype=np.float32).copy()
    lib().orc_shift_zerofill(_p(y, C.c_float), y.size, int(s))
    return y


def c_rfft(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros(x.size + 2, np.float32)
    if lib().orc_rfft_f32(x.size, _p(x, C.c_float), _p(out, C.c_float)) != 0:
        raise ValueError("rfft length must be a power of two")
    return out.view(np.complex64)


def c_irfft(s: np.ndarray, n: int) -> np.ndarray:
    s = np.ascontiguousarray(s, dtype=np.complex64)
    out = np.zeros(n, np.float32)
    lib().orc_irfft_f32(n, _p(s.view(np.float32), C.c_float), _p(out, C.c_float))
    return out


def c_delay_entries(scan: Scan, first: int, nf: int):
    cfg = scan.to_c()
    out = np.zeros(nf, dtype=[("int1", "<i8"), ("int2", "<i8"), ("frac1", "<f8"),
                              ("frac2", "<f8"), ("fr_lo1", "<f4", 2), ("fr_lo2", "<f4", 2)])
    fd = FrameDelay()
    for i in range(nf):
        lib().orc_delay_entry(C.byref(cfg.delay), first + i, C.byref(fd))
        out[i] = (fd.int1, fd.int2, fd.frac1, fd.frac2, tuple(fd.fr_lo1), tuple(fd.fr_lo2))
    return out


def c_band_alignment(fft, fs, c1, c2, bw1, bw2):
    out = (C.c_int64 * 4)()
    if lib().orc_band_alignment(fft, fs, c1, c2, bw1, bw2, out) != 0:
        raise ValueError("No band overlap")
    return tuple(out)


def c_quantise(samples: np.ndarray, bits: int, levels, shuffle_out) -> bytes:
    s = np.ascontiguousarray(samples, dtype=np.float32)
    cap = (s.size * bits + 31) // 32 * 4 + 4
    out = np.zeros(cap, np.uint8)
    lv = np.asarray(levels, np.float64)
    sh = np.asarray(shuffle_out, np.uint8)
    n = lib().orc_quantise_frame(_p(s, C.c_float), s.size, bits, _p(lv, C.c_double), lv.size,
                                 _p(sh, C.c_uint8), _p(out, C.c_uint8), cap)
    return out[:n].tobytes()


def c_sector_corr(scan: Scan, raw1, raw2, nf: int, first_frame: int = 0, nthreads: int = 0):
    cfg = scan.to_c()
    h = scan.h
    a11, a22 = np.zeros(h), np.zeros(h)
    a12 = np.zeros(2 * h)
    r1 = np.ascontiguousarray(raw1, dtype=np.uint8)
    r2 = np.ascontiguousarray(raw2, dtype=np.uint8)
    failed = lib().orc_sector_corr(C.byref(cfg), _p(r1, C.c_uint8), _p(r2, C.c_uint8), nf,
                                   first_frame, _p(a11, C.c_double), _p(a22, C.c_double),
                                   _p(a12, C.c_double), nthreads)
    return dict(acf11=a11, acf22=a22, xcf=a12.view(np.complex128), failed=failed)


def c_sector_phased(scan: Scan, raw1, raw2, nf: int, first_frame: int = 0, want_raw=True,
                    nthreads: int = 0):
    cfg = scan.to_c()
    ph = np.zeros(scan.h)
    r1 = np.ascontiguousarray(raw1, dtype=np.uint8)
    r2 = np.ascontiguousarray(raw2, dtype=np.uint8)
    out = np.zeros(nf * scan.bpf(scan.bits_out), np.uint8) if want_raw else None
    failed = lib().orc_sector_phased(C.byref(cfg), _p(r1, C.c_uint8), _p(r2, C.c_uint8), nf,
                                     first_frame, _p(ph, C.c_double),
                                     _p(out, C.c_uint8) if want_raw else None, nthreads)
    return dict(phased=ph, raw=out, failed=failed)


def c_normalize(fft, nf, level_power, acc_real=None, acc_cplx=None):
    out = np.zeros(fft, np.float32)
    ar = None if acc_real is None else np.ascontiguousarray(acc_real, np.float64)
    ac = None if acc_cplx is None else np.ascontiguousarray(
        np.asarray(acc_cplx, np.complex128).view(np.float64))
    lib().orc_normalize(fft, nf, level_power, None if ar is None else _p(ar, C.c_double),
                        None if ac is None else _p(ac, C.c_double), _p(out, C.c_float))
    return out.view(np.complex64)


def level_power(levels) -> float:
    """main.rs:378-387"""
    return sum(v * v for v in levels) / len(levels)


# ------------------------------------------------------ NumPy restatement

def np_shuffle_words(words: np.ndarray, shuffle) -> np.ndarray:
    """utils.rs:159-171 vectorised: out bit o = word bit shuffle[o]."""
    sh = list(shuffle)
    if sh == list(range(32)):
        return words
    out = np.zeros_like(words)
    for o in range(32):
        out |= ((words >> np.uint32(sh[o])) & np.uint32(1)) << np.uint32(o)
    return out


def np_decode_frames(raw: np.ndarray, nf: int, fft: int, bits: int, shuffle, levels, lsb: bool,
                     dtype=np.float64) -> np.ndarray:
    """Vectorised utils.rs:215-376 for whole frames (fft*bits a multiple of 32)."""
    assert (fft * bits) % 32 == 0
    bpf = fft * bits // 8
    b = np.ascontiguousarray(raw[: nf * bpf], dtype=np.uint8).reshape(nf, bpf)
    words = b.view("<u4").astype(np.uint32)
    words = np_shuffle_words(words, shuffle)
    per = 32 // bits
    shifts = (np.arange(per, dtype=np.uint32) * np.uint32(bits))
    codes = (words[:, :, None] >> shifts[None, None, :]) & np.uint32((1 << bits) - 1)
    codes = codes.reshape(nf, fft)
    lv = np.asarray(levels, dtype=dtype)
    x = lv[codes]
    if lsb:
        x[:, 1::2] *= -1
    return x


def np_shift_frames(x: np.ndarray, shifts: np.ndarray) -> np.ndarray:
    """utils.rs:126-145 per frame (rows of x)."""
    nf, n = x.shape
    y = np.zeros_like(x)
    for i in range(nf):
        s = int(shifts[i])
        if s == 0:
            y[i] = x[i]
        elif abs(s) >= n:
            pass
        elif s > 0:
            y[i, s:] = x[i, : n - s]
        else:
            y[i, : n + s] = x[i, -s:]
    return y


def np_delay_entries(scan: Scan, first: int, nf: int):
    """main.rs:184-241 in float64 (Python floats are IEEE doubles; the
    expression order follows the reference so integer shifts match).  The
    fringe phasor is left in float64 (no f32 cast) for the FP64 oracle."""
    d = scan.delay_cfg_dict()
    gt = scan.geom_table
    fs = d["fs"]
    out = []
    two_pi = 2.0 * math.pi
    for fi in range(first, first + nf):
        t_mid_local = (float(fi) + 0.5) * d["frame_dt"]
        t_mid = t_mid_local + d["time_offset_s"]
        if gt is not None:
            last = max(len(gt) - 1, 0)
            fl = math.floor(t_mid_local)
            sec = int(fl) if fl > 0.0 else 0
            i0 = min(sec, last)
            i1 = min(i0 + 1, last)
            frac = 0.0 if i1 == i0 else min(max(t_mid_local - float(i0), 0.0), 1.0)
            gd_t = float(gt[i0]) * (1.0 - frac) + float(gt[i1]) * frac
            net = gd_t + d["coarse_delay_s"] + d["delay_user_samples"] / fs + \
                d["extra_delay_rate_sps"] * t_mid
            c1 = d["clock1_delay_s"] + d["clock1_rate_sps"] * t_mid
            c2 = d["clock2_delay_s"] + d["clock2_rate_sps"] * t_mid
            full = net + (c2 - c1)
            tau1, tau2, t1f, t2f = full - d["d_seek"], 0.0, full, 0.0
        else:
            tau1 = d["net_d1_base"] + d["total_rate1_base"] * t_mid + \
                0.5 * d["total_accel1_base"] * (t_mid * t_mid)
            tau2 = d["net_d2_base"] + d["total_rate2_base"] * t_mid + \
                0.5 * d["total_accel2_base"] * (t_mid * t_mid)
            t1f, t2f = tau1 + d["d_seek"], tau2

        def split(tau):
            v = tau * fs
            a = abs(v)
            r = math.floor(a)
            if a - r >= 0.5:  # f64::round: half away from zero (a - r is exact)
                r += 1.0
            i = int(math.copysign(r, v))
            return i, tau - (float(i) / fs)

        def carrier(f, tau):
            if f == 0.0:
                return 0.0
            ph = -two_pi * f * tau
            m = math.fmod(ph + math.pi, two_pi)  # f64::rem_euclid
            if m < 0.0:
                m += abs(two_pi)
            return m - math.pi

        i1, f1 = split(tau1)
        i2, f2 = split(tau2)
        out.append((i1, i2, f1, f2, carrier(d["lo1_hz"], t1f), carrier(d["lo2_hz"], t2f)))
    return out


def fp64_sector_corr(scan: Scan, raw1, raw2, nf: int, first_frame: int = 0, chunk: int = 256):
    """FP64 oracle for one sector of the corr path (main.rs:2413-2591)."""
    n, h = scan.fft, scan.h
    sb, a1s, a1e, a2s = scan.band_or_default()
    ov = a1e - a1s
    df = scan.fs / n
    acc11, acc22 = np.zeros(h), np.zeros(h)
    acc12 = np.zeros(h, np.complex128)
    ents = np_delay_entries(scan, first_frame, nf)
    bpf1, bpf2 = scan.bpf(scan.bits1), scan.bpf(scan.bits2)
    overlap_only = bool(scan.products & PROD_ACF_OVERLAP_ONLY)
    k = np.arange(ov, dtype=np.float64)
    for c0 in range(0, nf, chunk):
        c1 = min(nf, c0 + chunk)
        m = c1 - c0
        x1 = np_decode_frames(raw1[c0 * bpf1:], m, n, scan.bits1, scan.shuffle1, scan.levels1,
                              scan.lsb1)
        x2 = np_decode_frames(raw2[c0 * bpf2:], m, n, scan.bits2, scan.shuffle2, scan.levels2,
                              scan.lsb2)
        e = ents[c0:c1]
        x1 = np_shift_frames(x1, np.array([t[0] for t in e]))
        x2 = np_shift_frames(x2, np.array([t[1] for t in e]))
        s1 = np.fft.rfft(x1, axis=1)
        s2 = np.fft.rfft(x2, axis=1)
        p1 = np.array([t[4] for t in e])
        p2 = np.array([t[5] for t in e])
        fr_mix = np.exp(1j * (p1 - p2))
        step1 = -2.0 * math.pi * df * np.array([t[2] for t in e])
        step2 = -2.0 * math.pi * df * np.array([t[3] for t in e])
        ramp = np.exp(1j * ((step1[:, None] * (a1s + k)[None, :]) -
                            (step2[:, None] * (a2s + k)[None, :])))
        o1 = s1[:, a1s:a1e]
        o2 = s2[:, a2s:a2s + ov]
        if scan.products & PROD_ACF:
            if scan.grid == 0:
                g = slice(a1s, a1e)
                if overlap_only:
                    acc11[g] += (np.abs(o1) ** 2).sum(0)
                else:
                    acc11 += (np.abs(s1) ** 2).sum(0)
                acc22[g] += (np.abs(o2) ** 2).sum(0)
            else:
                g = slice(a2s, a2s + ov)
                if overlap_only:
                    acc22[g] += (np.abs(o2) ** 2).sum(0)
                else:
                    acc22 += (np.abs(s2) ** 2).sum(0)
                acc11[g] += (np.abs(o1) ** 2).sum(0)
        if scan.products & PROD_XCF:
            v = (o1 * np.conj(o2) * fr_mix[:, None] * ramp).sum(0)
            if scan.grid == 0:
                acc12[a1s:a1e] += v
            else:
                acc12[a2s:a2s + ov] += v
    return dict(acf11=acc11, acf22=acc22, xcf=acc12, failed=0)


def fp64_sector_corr_parallel(scan: Scan, raw1, raw2, nf: int, first_frame: int = 0,
                              workers: int = 0, pieces_per_worker: int = 4):
    """fp64_sector_corr over contiguous frame ranges in worker processes,
    summed in range order: the FP64 oracle for sectors of 1e9 samples.  The
    pool uses the spawn start method, which is safe in a process that has
    already initialised CUDA (a forked child of such a process can hang)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    workers = workers or os.cpu_count() or 1
    npieces = max(1, min(nf, workers * pieces_per_worker))
    bounds = [nf * k // npieces for k in range(npieces + 1)]
    b1, b2 = scan.bpf(scan.bits1), scan.bpf(scan.bits2)
    r1 = np.asarray(raw1, np.uint8)
    r2 = np.asarray(raw2, np.uint8)
    total = None
    with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        futs = [ex.submit(fp64_sector_corr, scan, r1[f0 * b1:f1 * b1], r2[f0 * b2:f1 * b2],
                          f1 - f0, first_frame + f0)
                for f0, f1 in zip(bounds[:-1], bounds[1:]) if f1 > f0]
        for f in futs:
            part = f.result()
            if total is None:
                total = part
            else:
                for k in ("acf11", "acf22", "xcf"):
                    total[k] = total[k] + part[k]
    return total


def fp64_sector_phased(scan: Scan, raw1, raw2, nf: int, first_frame: int = 0, chunk: int = 256):
    """FP64 oracle for the phased power of one sector (main.rs:2222-2365),
    plus the float64 time series that the .raw output quantises."""
    n, h = scan.fft, scan.h
    sb, a1s, a1e, a2s = scan.band_or_default()
    ov = a1e - a1s
    df = scan.fs / n
    acc = np.zeros(h)
    ents = np_delay_entries(scan, first_frame, nf)
    bpf1, bpf2 = scan.bpf(scan.bits1), scan.bpf(scan.bits2)
    kk = np.arange(h, dtype=np.float64)
    series = []
    for c0 in range(0, nf, chunk):
        c1 = min(nf, c0 + chunk)
        m = c1 - c0
        x1 = np_decode_frames(raw1[c0 * bpf1:], m, n, scan.bits1, scan.shuffle1, scan.levels1,
                              scan.lsb1)
        x2 = np_decode_frames(raw2[c0 * bpf2:], m, n, scan.bits2, scan.shuffle2, scan.levels2,
                              scan.lsb2)
        e = ents[c0:c1]
        x1 = np_shift_frames(x1, np.array([t[0] for t in e]))
        x2 = np_shift_frames(x2, np.array([t[1] for t in e]))
        s1 = np.fft.rfft(x1, axis=1)
        s2 = np.fft.rfft(x2, axis=1)
        f1 = np.array([t[2] for t in e])
        f2 = np.array([t[3] for t in e])
        s1 = s1 * np.exp(-2j * math.pi * df * f1[:, None] * kk[None, :])
        s2 = s2 * np.exp(-2j * math.pi * df * f2[:, None] * kk[None, :])
        s1[:, n // 2] = s1[:, n // 2].real
        s2[:, n // 2] = s2[:, n // 2].real
        s1 = s1 * np.exp(1j * np.array([t[4] for t in e]))[:, None]
        s2 = s2 * np.exp(1j * np.array([t[5] for t in e]))[:, None]
        cb = np.zeros((m, h), np.complex128)
        if scan.grid == 0:
            cb += s1 * scan.w1
            cb[:, a1s:a1e] += s2[:, a2s:a2s + ov] * scan.w2
        else:
            cb += s2 * scan.w2
            cb[:, a2s:a2s + ov] += s1[:, a1s:a1e] * scan.w1
        acc += (np.abs(cb) ** 2).sum(0)
        cb[:, 0] = cb[:, 0].real
        cb[:, n // 2] = cb[:, n // 2].real
        t = np.fft.irfft(cb, n=n, axis=1)
        if scan.lsb1 and scan.lsb2:
            t[:, 1::2] *= -1
        series.append(t)
    return dict(phased=acc, series=np.concatenate(series, 0) if series else None)


# --------------------------------------------------------- synthetic data

def pack_codes(codes: np.ndarray, bits: int, shuffle) -> np.ndarray:
    """Pack codes LSB-first into LE u32 words and apply the shuffle inverse
    (utils.rs:390-398 quantise_frame packing with shuffle_out = shuffle)."""
    codes = np.asarray(codes, dtype=np.uint32).reshape(-1)
    per = 32 // bits
    assert codes.size % per == 0
    cw = codes.reshape(-1, per)
    shifts = np.arange(per, dtype=np.uint32) * np.uint32(bits)
    words = np.bitwise_or.reduce(cw << shifts[None, :], axis=1).astype(np.uint32)
    sh = list(shuffle)
    if sh != list(range(32)):
        out = np.zeros_like(words)
        for pos in range(32):
            out |= ((words >> np.uint32(pos)) & np.uint32(1)) << np.uint32(sh[pos])
        words = out
    return words.astype("<u4").view(np.uint8)


def quantise_codes(x: np.ndarray, levels) -> np.ndarray:
    """Nearest-level code (first index wins ties), utils.rs:384-389."""
    lv = np.asarray(levels, np.float32)
    err = np.abs(x.astype(np.float32)[..., None] - lv[None, :])
    return np.argmin(err, axis=-1).astype(np.uint32)


def default_levels(bits: int):
    """Level tables used by the synthetic configs: 1-bit ±1, 2-bit ±1/±3,
    4- and 8-bit uniform half-integer steps (8-bit spans ±127.5)."""
    if bits == 1:
        return [-1.0, 1.0]
    if bits == 2:
        return [-3.0, -1.0, 1.0, 3.0]
    m = 1 << bits
    return [float(i) - (m - 1) / 2.0 for i in range(m)]


def level_gain(bits: int) -> float:
    """Gain applied to unit-variance noise before nearest-level quantisation:
    2-bit puts the ±2 decision points at ±0.98 sigma; wider words use a
    step of about sigma/ (2^(b-1)/3.5)."""
    if bits == 1:
        return 1.0
    if bits == 2:
        return 2.0 / 0.98
    return (1 << (bits - 1)) / 3.5


def synth_station_pair(n_samples: int, seed: int, rho: float = 0.05, delay_samples: float = 0.0,
                       tone_bin=None, tone_db: float = -30.0, fft: int = 1024):
    """Seeded Gaussian streams x1, x2 (unit variance) sharing a common
    component of fractional correlation rho; the common part reaching station
    2 is delayed by ``delay_samples`` (integer + fractional, applied in the
    frequency domain on the whole block).  Optional tone at FFT bin
    ``tone_bin`` (of an ``fft``-point frame) at ``tone_db`` below the noise."""
    rng = np.random.Generator(np.random.PCG64(seed))
    c = rng.standard_normal(n_samples)
    n1 = rng.standard_normal(n_samples)
    n2 = rng.standard_normal(n_samples)
    if delay_samples != 0.0:
        f = np.fft.rfftfreq(n_samples)
        c2 = np.fft.irfft(np.fft.rfft(c) * np.exp(-2j * np.pi * f * delay_samples), n=n_samples)
    else:
        c2 = c
    a, b = math.sqrt(rho), math.sqrt(1.0 - rho)
    x1 = a * c + b * n1
    x2 = a * c2 + b * n2
    if tone_bin is not None:
        amp = math.sqrt(2.0) * 10 ** (tone_db / 20.0)
        t = np.arange(n_samples)
        ph = rng.uniform(0, 2 * np.pi)
        tone = amp * np.cos(2 * np.pi * tone_bin * t / fft + ph)
        x1 = x1 + tone
        x2 = x2 + tone
    return x1, x2


def encode_station(x: np.ndarray, bits: int, levels, shuffle, lsb: bool, gain=None) -> np.ndarray:
    """Quantise a float series to codes and pack it into the .raw layout the
    decoder reads (LSB stations get odd samples negated, which the decoder
    undoes)."""
    g = level_gain(bits) if gain is None else gain
    y = np.asarray(x, np.float64) * g
    if lsb:
        y = y.copy()
        y[1::2] *= -1
    return pack_codes(quantise_codes(y, levels), bits, shuffle)


def synth_packed_pair(n_samples: int, seed: int, bits: int, levels, shuffle1, lsb1: bool,
                      shuffle2, lsb2: bool, rho: float = 0.05, lag: int = 7, gain=None,
                      nthreads: int = 0, tone_bin=None, tone_db: float = -30.0, fft: int = 1024):
    """Both stations' packed .raw bytes of seeded quantised Gaussian noise
    (common component at rho, station 2 `lag` whole samples late; optionally
    a tone at FFT bin `tone_bin` of an `fft`-point frame, `tone_db` below the
    noise, at both stations, as synth_station_pair adds it), written by
    the C generator in synth.c: fast enough for full-size sectors (1e9
    samples per station in seconds), identical for any thread count.  The
    shuffles are the stations' internal maps, applied inversely as the
    encoder above does."""
    g = level_gain(bits) if gain is None else gain
    lv = np.ascontiguousarray(levels, np.float64)
    s1 = np.ascontiguousarray(shuffle1, np.uint8)
    s2 = np.ascontiguousarray(shuffle2, np.uint8)
    nb = n_samples * bits // 8
    o1, o2 = np.empty(nb, np.uint8), np.empty(nb, np.uint8)
    nt = nthreads or os.cpu_count() or 1
    amp = 0.0 if tone_bin is None else math.sqrt(2.0) * 10 ** (tone_db / 20.0)
    cyc = 0.0 if tone_bin is None else tone_bin / fft
    ph = 0.0 if tone_bin is None else float(np.random.Generator(np.random.PCG64(seed)).uniform(
        0, 2 * np.pi))
    rc = lib().orc_synth_pack_pair(seed, n_samples, rho, lag, amp, cyc, ph, bits,
                                   _p(lv, C.c_double), lv.size,
                                   g, _p(s1, C.c_uint8), int(lsb1), _p(s2, C.c_uint8), int(lsb2),
                                   _p(o1, C.c_uint8), _p(o2, C.c_uint8), nt)
    if rc != 0:
        raise ValueError("orc_synth_pack_pair: bad arguments")
    return o1, o2


def random_shuffle(seed: int, avoid_special: bool = True):
    rng = np.random.Generator(np.random.PCG64(seed))
    while True:
        p = [int(v) for v in rng.permutation(32)]
        if not avoid_special or (p != list(range(32)) and p != [i ^ 1 for i in range(32)]):
            return p
