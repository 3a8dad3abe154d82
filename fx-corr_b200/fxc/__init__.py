"""fxc — Python binding of libfxc.so, the B200 FX-correlation engine.

Everything here goes through the C ABI declared in include/fxc.h (ctypes, plain
pointers and sizes).  PyTorch is used only to hold device buffers and to hand
CUDA stream handles to the library; the computation is the library's CUDA
kernels.  There is no CPU fallback: if libfxc.so is missing or the device is
not an sm_100 part, calls raise.

Reference: fx-corr (Rust CPU correlator); the per-sector call replaces the
body of the sector loop in src/main.rs:2173-2683.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libfxc.so"
HEADER = PKG.parent.parent / "include" / "fxc.h"

OK, EINVAL, ENOMEM, ECUDA, ETIMEDOUT, ENOTFOUND, EBUSY, EUNSUPPORTED, EDEVICE = (
    0, -1, -2, -3, -4, -5, -6, -7, -8)
PROD_ACF, PROD_XCF, PROD_PHASED, PROD_RAW, PROD_ACF_OVERLAP_ONLY = 1, 2, 4, 8, 16

# Every function include/fxc.h declares (checked by the CPU test suite).
EXPORTS = [
    "fxc_abi_version", "fxc_status_string", "fxc_last_error", "fxc_engine_create",
    "fxc_engine_destroy", "fxc_scan_open", "fxc_scan_close", "fxc_sector_submit",
    "fxc_sector_wait", "fxc_sector_run_device", "fxc_scan_check", "fxc_delay_entries_device",
    "fxc_decode_device", "fxc_spectra_device", "fxc_parse_shuffle", "fxc_band_alignment",
    "fxc_level_power", "fxc_normalize", "fxc_bytes_per_frame", "fxc_probe_fp32_peak",
    "fxc_scan_set_profiling", "fxc_scan_profile", "fxc_sector_run_device_noalloc",
    "fxc_server_create", "fxc_server_submit", "fxc_server_wait", "fxc_server_destroy",
    "fxc_host_alloc", "fxc_host_free", "fxc_batch_create", "fxc_batch_destroy",
    "fxc_batch_run_device", "fxc_batch_autotune", "fxc_batch_shape", "fxc_batch_launches",
    "fxc_batch_set_shape", "fxc_sector_noalloc_check", "fxc_debug_inject_wait_timeout",
    "fxc_host_register", "fxc_host_unregister", "fxc_batch_run_device_raw",
    "fxc_probe_exchange", "fxc_probe_mma_f16",
]
NOALLOC_MAX_FRAMES = 32768


class FxcError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"fxc status {status}: {msg}")
        self.status = status


# ------------------------------------------------------------------ structs

class DelayCfg(C.Structure):
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
    _fields_ = [("int1", C.c_int64), ("int2", C.c_int64), ("frac1", C.c_double),
                ("frac2", C.c_double), ("fr_lo1", C.c_float * 2), ("fr_lo2", C.c_float * 2)]


FRAME_DELAY_DTYPE = np.dtype([("int1", "<i8"), ("int2", "<i8"), ("frac1", "<f8"),
                              ("frac2", "<f8"), ("fr_lo1", "<f4", 2), ("fr_lo2", "<f4", 2)])


class ScanCfgC(C.Structure):
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


class DeviceOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_inflight", C.c_int32),
                ("hbm_budget_bytes", C.c_uint64)]


class ServerOpts(C.Structure):
    _fields_ = [("slots", C.c_int32), ("batch", C.c_int32)]


class BatchOpts(C.Structure):
    _fields_ = [("use_graphs", C.c_int32), ("autotune", C.c_int32), ("item_frames", C.c_uint32)]


class JobC(C.Structure):
    _fields_ = [("cfg", C.c_void_p), ("raw1", C.c_void_p), ("raw2", C.c_void_p),
                ("nf", C.c_uint64), ("first_frame", C.c_uint64), ("sector_frames", C.c_uint64),
                ("out", C.c_void_p), ("raw_out", C.c_void_p)]


class JobStats(C.Structure):
    _fields_ = [("status", C.c_int32), ("sectors", C.c_uint32), ("t_submit_ns", C.c_uint64),
                ("t_start_ns", C.c_uint64), ("t_done_ns", C.c_uint64)]


class SectorOut(C.Structure):
    _fields_ = [("acf11", C.POINTER(C.c_double)), ("acf22", C.POINTER(C.c_double)),
                ("xcf", C.POINTER(C.c_double)), ("phased", C.POINTER(C.c_double)),
                ("raw_out", C.POINTER(C.c_uint8)), ("raw_out_len", C.c_uint64),
                ("frames_failed", C.c_uint64)]


# ---------------------------------------------------------------- loading

_lib = None


def lib():
    """Load libfxc.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FxcError(EUNSUPPORTED, f"{LIB_PATH} is not built (run fxc.build.build())")
    L = C.CDLL(str(LIB_PATH))
    vp, u8p, f32p, f64p = C.c_void_p, C.POINTER(C.c_uint8), C.c_void_p, C.POINTER(C.c_double)
    st = C.c_int32
    sig = {
        "fxc_abi_version": ([], C.c_int32),
        "fxc_status_string": ([st], C.c_char_p),
        "fxc_last_error": ([], C.c_char_p),
        "fxc_engine_create": ([C.POINTER(DeviceOpts), C.POINTER(vp)], st),
        "fxc_engine_destroy": ([vp], st),
        "fxc_scan_open": ([vp, C.POINTER(ScanCfgC), C.POINTER(vp)], st),
        "fxc_scan_close": ([vp], st),
        "fxc_sector_submit": ([vp, vp, C.c_uint64, vp, C.c_uint64, C.c_uint64, C.c_uint64,
                               C.POINTER(C.c_uint64)], st),
        "fxc_sector_wait": ([vp, C.c_uint64, C.c_int32, C.POINTER(SectorOut)], st),
        "fxc_sector_run_device": ([vp, vp, vp, C.c_uint64, C.c_uint64, vp, vp, vp], st),
        "fxc_scan_check": ([vp], st),
        "fxc_delay_entries_device": ([vp, C.c_uint64, C.c_uint64, vp, vp], st),
        "fxc_decode_device": ([vp, vp, vp, C.c_uint64, C.c_uint64, vp, vp, vp], st),
        "fxc_spectra_device": ([vp, vp, vp, C.c_uint64, C.c_uint64, vp, vp, vp], st),
        "fxc_parse_shuffle": ([C.POINTER(C.c_int32), u8p], st),
        "fxc_band_alignment": ([C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_double,
                                C.c_double, C.POINTER(C.c_int64)], st),
        "fxc_level_power": ([f64p, C.c_uint32, f64p], st),
        "fxc_normalize": ([C.c_uint32, C.c_uint64, C.c_double, f64p, f64p, vp], st),
        "fxc_bytes_per_frame": ([C.c_uint32, C.c_uint32], C.c_uint64),
        "fxc_probe_fp32_peak": ([C.c_int32, f64p], st),
        "fxc_probe_exchange": ([C.c_int32, f64p, f64p], st),
        "fxc_probe_mma_f16": ([C.c_int32, f64p], st),
        "fxc_scan_set_profiling": ([vp, C.c_int32], st),
        "fxc_sector_run_device_noalloc": ([C.POINTER(ScanCfgC), vp, vp, C.c_uint64, C.c_uint64,
                                           vp, vp], st),
        "fxc_sector_noalloc_check": ([vp], st),
        "fxc_debug_inject_wait_timeout": ([C.c_uint32, C.c_int32], st),
        "fxc_scan_profile": ([vp, f64p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_int32],
                             st),
        "fxc_server_create": ([vp, C.POINTER(ServerOpts), C.POINTER(vp)], st),
        "fxc_server_submit": ([vp, C.POINTER(JobC), C.POINTER(C.c_uint64)], st),
        "fxc_server_wait": ([vp, C.c_uint64, C.c_int32, C.POINTER(JobStats)], st),
        "fxc_server_destroy": ([vp], st),
        "fxc_host_alloc": ([C.c_uint64, C.POINTER(vp)], st),
        "fxc_host_free": ([vp], st),
        "fxc_host_register": ([vp, C.c_uint64], st),
        "fxc_host_unregister": ([vp], st),
        "fxc_batch_create": ([vp, C.POINTER(BatchOpts), C.POINTER(vp)], st),
        "fxc_batch_destroy": ([vp], st),
        "fxc_batch_run_device": ([vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(vp),
                                  C.c_uint32, vp], st),
        "fxc_batch_run_device_raw": ([vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                      C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                      C.POINTER(vp), C.POINTER(vp), C.c_uint32, vp], st),
        "fxc_batch_autotune": ([vp, C.c_uint32], st),
        "fxc_batch_shape": ([vp, C.c_uint32, C.POINTER(C.c_int32), C.POINTER(C.c_uint32),
                             C.POINTER(C.c_int32), f64p], st),
        "fxc_batch_launches": ([vp], C.c_uint64),
        "fxc_batch_set_shape": ([vp, C.c_uint32, C.c_int32, C.c_uint32], st),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def check(status: int):
    if status != OK:
        msg = lib().fxc_last_error().decode(errors="replace")
        raise FxcError(status, msg or lib().fxc_status_string(status).decode())


def _ptr(t) -> int:
    """Device or host address of a torch tensor / numpy array (None -> 0)."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def _stream(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


# --------------------------------------------------------------- config

@dataclass
class ScanConfig:
    """Per-scan configuration (fields of fxc_scan_cfg).  ``band`` is
    (shift_bins, a1s, a1e, a2s); None means no band shift over bins
    [0, fft/2).  ``delay`` holds DelayEvalConfig fields (src/main.rs:161-182);
    ``geom_table`` the optional 1-s geometric-delay table."""

    fft: int = 1024
    fs: float = 32e6
    bits1: int = 2
    bits2: int = 2
    levels1: list = field(default_factory=lambda: [-1.5, -0.5, 0.5, 1.5])
    levels2: list = field(default_factory=lambda: [-1.5, -0.5, 0.5, 1.5])
    shuffle1: list = field(default_factory=lambda: list(range(32)))
    shuffle2: list = field(default_factory=lambda: list(range(32)))
    lsb1: bool = False
    lsb2: bool = False
    band: tuple = None
    grid: int = 0
    products: int = PROD_ACF | PROD_XCF
    w1: float = 1.0
    w2: float = 1.0
    delay: dict = field(default_factory=dict)
    geom_table: object = None

    @property
    def h(self):
        return self.fft // 2 + 1

    @property
    def bits_out(self):
        return max(self.bits1, self.bits2)

    def bpf(self, bits):
        return int(lib().fxc_bytes_per_frame(self.fft, bits))

    def to_c(self) -> ScanCfgC:
        c = ScanCfgC()
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
        sb, a1s, a1e, a2s = self.band if self.band is not None else (0, 0, self.fft // 2, 0)
        c.shift_bins, c.a1s, c.a1e, c.a2s = sb, a1s, a1e, a2s
        c.grid, c.products, c.w1, c.w2 = self.grid, self.products, self.w1, self.w2
        d = dict(frame_dt=self.fft / self.fs, fs=self.fs)
        d.update(self.delay)
        for k, v in d.items():
            setattr(c.delay, k, v)
        if self.geom_table is not None:
            self._gt = np.ascontiguousarray(self.geom_table, dtype=np.float64)
            c.delay.geom_table = self._gt.ctypes.data_as(C.POINTER(C.c_double))
            c.delay.geom_len = len(self._gt)
        return c


# ---------------------------------------------------------------- objects

class Engine:
    def __init__(self, device: int = 0, max_inflight: int = 2, hbm_budget_bytes: int = 0):
        o = DeviceOpts(device, max_inflight, hbm_budget_bytes)
        h = C.c_void_p()
        check(lib().fxc_engine_create(C.byref(o), C.byref(h)))
        self.h = h
        self.device = device
        self._scans = weakref.WeakSet()
        self._servers = weakref.WeakSet()
        self._batches = weakref.WeakSet()

    def open_scan(self, cfg: ScanConfig) -> "Scan":
        s = Scan(self, cfg)
        self._scans.add(s)
        return s

    def close(self):
        if self.h:
            # the library destroys the engine's servers and closes its scans
            for s in list(self._scans):
                s.h = None
            for sv in list(self._servers):
                sv.h = None
            for b in list(self._batches):
                b.h = None
            lib().fxc_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scan:
    def __init__(self, eng: Engine, cfg: ScanConfig):
        self.eng, self.cfg = eng, cfg
        c = cfg.to_c()
        h = C.c_void_p()
        check(lib().fxc_scan_open(eng.h, C.byref(c), C.byref(h)))
        self.h = h

    def close(self):
        if self.h and self.eng.h:
            lib().fxc_scan_close(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- device-resident path
    def run_device(self, d_raw1, d_raw2, nf: int, first_frame: int, d_acc, d_raw_out=None,
                   stream=None):
        check(lib().fxc_sector_run_device(self.h, _ptr(d_raw1), _ptr(d_raw2), nf, first_frame,
                                          _ptr(d_acc), _ptr(d_raw_out), _stream(stream)))

    def check(self):
        check(lib().fxc_scan_check(self.h))

    def set_profiling(self, enable: bool = True):
        check(lib().fxc_scan_set_profiling(self.h, int(enable)))

    def profile(self, reset: bool = False):
        """(correlation-kernel device ms, its launches, all library launches)."""
        ms, kl, al = C.c_double(), C.c_uint64(), C.c_uint64()
        check(lib().fxc_scan_profile(self.h, C.byref(ms), C.byref(kl), C.byref(al), int(reset)))
        return ms.value, kl.value, al.value

    def delay_entries(self, first_frame: int, nf: int, stream=None):
        import torch
        out = torch.empty(nf * FRAME_DELAY_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        check(lib().fxc_delay_entries_device(self.h, first_frame, nf, _ptr(out), _stream(stream)))
        torch.cuda.synchronize()
        return out.cpu().numpy().view(FRAME_DELAY_DTYPE)

    def decode(self, d_raw1, d_raw2, nf: int, first_frame: int = 0, stream=None):
        import torch
        x1 = torch.empty(nf * self.cfg.fft, dtype=torch.float32, device="cuda")
        x2 = torch.empty_like(x1)
        check(lib().fxc_decode_device(self.h, _ptr(d_raw1), _ptr(d_raw2), nf, first_frame,
                                      _ptr(x1), _ptr(x2), _stream(stream)))
        return x1.view(nf, self.cfg.fft), x2.view(nf, self.cfg.fft)

    def spectra(self, d_raw1, d_raw2, nf: int, first_frame: int = 0, stream=None):
        import torch
        h = self.cfg.h
        s1 = torch.empty(nf * h * 2, dtype=torch.float32, device="cuda")
        s2 = torch.empty_like(s1)
        check(lib().fxc_spectra_device(self.h, _ptr(d_raw1), _ptr(d_raw2), nf, first_frame,
                                       _ptr(s1), _ptr(s2), _stream(stream)))
        return (torch.view_as_complex(s1.view(nf, h, 2)), torch.view_as_complex(s2.view(nf, h, 2)))

    def sector_device(self, d_raw1, d_raw2, nf: int, first_frame: int = 0, stream=None):
        """Run one sector on device inputs; returns the host result dict."""
        import torch
        h = self.cfg.h
        acc = torch.empty(5 * h, dtype=torch.float64, device="cuda")
        raw = None
        if self.cfg.products & PROD_RAW:
            raw = torch.empty(max(1, nf * self.cfg.bpf(self.cfg.bits_out)), dtype=torch.uint8,
                              device="cuda")
        self.run_device(d_raw1, d_raw2, nf, first_frame, acc, d_raw_out=raw, stream=stream)
        self.check()
        a = acc.cpu().numpy()
        out = dict(acf11=a[:h], acf22=a[h:2 * h], xcf=a[2 * h:4 * h].view(np.complex128),
                   phased=a[4 * h:])
        if raw is not None:
            out["raw"] = raw.cpu().numpy()[: nf * self.cfg.bpf(self.cfg.bits_out)]
        return out

    # -- host-buffer path (the reference-facing per-sector call)
    def submit(self, raw1, raw2, nf: int, first_frame: int = 0) -> int:
        r1 = np.ascontiguousarray(raw1, dtype=np.uint8)
        r2 = np.ascontiguousarray(raw2, dtype=np.uint8)
        sid = C.c_uint64()
        check(lib().fxc_sector_submit(self.h, r1.ctypes.data, r1.size, r2.ctypes.data, r2.size,
                                      nf, first_frame, C.byref(sid)))
        self._keep = getattr(self, "_keep", {})
        self._keep[sid.value] = (r1, r2)
        self._nf = getattr(self, "_nf", {})
        self._nf[sid.value] = nf
        return sid.value

    def wait(self, sector_id: int, timeout_ms: int = -1) -> dict:
        h = self.cfg.h
        a11, a22, ph = np.zeros(h), np.zeros(h), np.zeros(h)
        x = np.zeros(2 * h)
        o = SectorOut()
        o.acf11 = a11.ctypes.data_as(C.POINTER(C.c_double))
        o.acf22 = a22.ctypes.data_as(C.POINTER(C.c_double))
        o.xcf = x.ctypes.data_as(C.POINTER(C.c_double))
        o.phased = ph.ctypes.data_as(C.POINTER(C.c_double))
        raw = None
        if self.cfg.products & PROD_RAW:
            nf = getattr(self, "_nf", {}).get(sector_id, 0)
            raw = np.zeros(max(1, nf * self.cfg.bpf(self.cfg.bits_out)), np.uint8)
            o.raw_out = raw.ctypes.data_as(C.POINTER(C.c_uint8))
            o.raw_out_len = raw.size
        try:
            check(lib().fxc_sector_wait(self.h, sector_id, timeout_ms, C.byref(o)))
        finally:
            getattr(self, "_keep", {}).pop(sector_id, None)
        out = dict(acf11=a11, acf22=a22, xcf=x.view(np.complex128), phased=ph,
                   failed=o.frames_failed)
        if raw is not None:
            out["raw"] = raw[: getattr(self, "_nf", {}).pop(sector_id, 0) *
                             self.cfg.bpf(self.cfg.bits_out)]
        return out


class Batch:
    """Batched sectors of many scans (fxc_batch_*): one sector of each scan in
    a few launches, optionally replayed from captured CUDA graphs, with kernel
    shapes from the autotuner."""

    def __init__(self, eng: Engine, use_graphs: bool = False, autotune: bool = False,
                 item_frames: int = 0):
        self.eng = eng
        h = C.c_void_p()
        o = BatchOpts(int(use_graphs), int(autotune), item_frames)
        check(lib().fxc_batch_create(eng.h, C.byref(o), C.byref(h)))
        self.h = h
        eng._batches.add(self)

    def run_device(self, scans, d_raw1, d_raw2, nf, first_frame, d_acc, stream=None):
        """One sector per scan; every argument but stream is a sequence of the
        same length (torch CUDA tensors for the buffers)."""
        n = len(scans)
        VP = C.c_void_p * n
        U64 = C.c_uint64 * n
        check(lib().fxc_batch_run_device(
            self.h, VP(*[s.h.value for s in scans]), VP(*[_ptr(x) for x in d_raw1]),
            VP(*[_ptr(x) for x in d_raw2]), U64(*nf), U64(*first_frame),
            VP(*[_ptr(x) for x in d_acc]), n, _stream(stream)))

    def run_device_raw(self, scans, d_raw1, d_raw2, nf, first_frame, d_acc, d_raw_out,
                       stream=None):
        """run_device with phased .raw outputs: d_raw_out[i] is a device buffer
        (or None) for scan i's re-quantised frames."""
        n = len(scans)
        VP = C.c_void_p * n
        U64 = C.c_uint64 * n
        check(lib().fxc_batch_run_device_raw(
            self.h, VP(*[s.h.value for s in scans]), VP(*[_ptr(x) for x in d_raw1]),
            VP(*[_ptr(x) for x in d_raw2]), U64(*nf), U64(*first_frame),
            VP(*[_ptr(x) for x in d_acc]), VP(*[_ptr(x) for x in d_raw_out]), n,
            _stream(stream)))

    def autotune(self, fft: int):
        check(lib().fxc_batch_autotune(self.h, fft))

    def shape(self, fft: int) -> dict:
        fpc, itf, ctas, g = C.c_int32(), C.c_uint32(), C.c_int32(), C.c_double()
        check(lib().fxc_batch_shape(self.h, fft, C.byref(fpc), C.byref(itf), C.byref(ctas),
                                    C.byref(g)))
        return dict(fpc=fpc.value, item_frames=itf.value, ctas_per_sm=ctas.value,
                    gsps=g.value)

    def set_shape(self, fft: int, fpc: int, item_frames: int):
        check(lib().fxc_batch_set_shape(self.h, fft, fpc, item_frames))

    def launches(self) -> int:
        return int(lib().fxc_batch_launches(self.h))

    def close(self):
        if self.h and self.eng.h:
            lib().fxc_batch_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The serving loop (fxc_server_*): jobs of one scan configuration each,
    admitted into ``slots`` concurrent device contexts as they free up."""

    def __init__(self, eng: Engine, slots: int = 4, batch: bool = False):
        self.eng = eng
        h = C.c_void_p()
        check(lib().fxc_server_create(eng.h, C.byref(ServerOpts(slots, int(batch))), C.byref(h)))
        self.h = h
        self._jobs = {}
        eng._servers.add(self)

    def submit(self, cfg: ScanConfig, raw1, raw2, nf: int, first_frame: int = 0,
               sector_frames: int = 0, cfg_c=None) -> int:
        """Queue a job; raw1/raw2 are host arrays (page-locked torch tensors
        or numpy arrays) that must stay alive until wait().  cfg_c: cfg.to_c()
        built beforehand (a caller submitting many jobs of few configurations)."""
        c = cfg.to_c() if cfg_c is None else cfg_c
        sf = sector_frames or max(nf, 1)
        nsec = (nf + sf - 1) // sf if nf else 1
        out = np.zeros((nsec, 5 * cfg.h))
        raw = None
        if cfg.products & PROD_RAW:
            raw = np.zeros(max(1, nf * cfg.bpf(cfg.bits_out)), np.uint8)
        j = JobC(C.addressof(c), _ptr(raw1), _ptr(raw2), nf, first_frame, sector_frames,
                 out.ctypes.data, None if raw is None else raw.ctypes.data)
        jid = C.c_uint64()
        check(lib().fxc_server_submit(self.h, C.byref(j), C.byref(jid)))
        self._jobs[jid.value] = (cfg, raw1, raw2, out, raw)
        return jid.value

    def wait(self, job_id: int, timeout_ms: int = -1):
        """(list of per-dump result dicts, stats dict) of a finished job."""
        st = JobStats()
        try:
            check(lib().fxc_server_wait(self.h, job_id, timeout_ms, C.byref(st)))
        except FxcError as e:
            if e.status != ETIMEDOUT:
                self._jobs.pop(job_id, None)
            raise
        cfg, _, _, out, raw = self._jobs.pop(job_id)
        h = cfg.h
        dumps = [dict(acf11=o[:h], acf22=o[h:2 * h], xcf=o[2 * h:4 * h].view(np.complex128),
                      phased=o[4 * h:]) for o in out]
        stats = dict(status=st.status, sectors=st.sectors, t_submit_ns=st.t_submit_ns,
                     t_start_ns=st.t_start_ns, t_done_ns=st.t_done_ns,
                     latency_s=(st.t_done_ns - st.t_submit_ns) * 1e-9)
        if raw is not None:
            stats["raw"] = raw
        return dumps, stats

    def close(self):
        if self.h and self.eng.h:
            lib().fxc_server_destroy(self.h)
        self.h = None
        self._jobs.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# -------------------------------------------------------------- helpers

def parse_shuffle(ext) -> list:
    e = (C.c_int32 * 32)(*ext)
    out = (C.c_uint8 * 32)()
    check(lib().fxc_parse_shuffle(e, out))
    return list(out)


def band_alignment(fft, fs, c1_mhz, c2_mhz, bw1_mhz, bw2_mhz):
    out = (C.c_int64 * 4)()
    check(lib().fxc_band_alignment(fft, fs, c1_mhz, c2_mhz, bw1_mhz, bw2_mhz, out))
    return tuple(out)


def level_power(levels) -> float:
    a = np.ascontiguousarray(levels, dtype=np.float64)
    out = C.c_double()
    check(lib().fxc_level_power(a.ctypes.data_as(C.POINTER(C.c_double)), a.size, C.byref(out)))
    return out.value


def normalize(fft, nf, level_power_, acc_real=None, acc_cplx=None):
    out = np.zeros(fft, np.float32)
    ar = None if acc_real is None else np.ascontiguousarray(acc_real, np.float64)
    ac = None if acc_cplx is None else np.ascontiguousarray(
        np.asarray(acc_cplx, np.complex128).view(np.float64))
    f64 = C.POINTER(C.c_double)
    check(lib().fxc_normalize(fft, nf, level_power_,
                              None if ar is None else ar.ctypes.data_as(f64),
                              None if ac is None else ac.ctypes.data_as(f64), out.ctypes.data))
    return out.view(np.complex64)


def sector_run_device_noalloc(cfg: ScanConfig, d_raw1, d_raw2, nf: int, first_frame: int,
                              d_acc, stream=None):
    """fxc_sector_run_device_noalloc: one sector on device inputs without any
    device allocation (scratch is the library's fixed array), on the current
    device; asynchronous on `stream`."""
    c = cfg.to_c()
    check(lib().fxc_sector_run_device_noalloc(C.byref(c), _ptr(d_raw1), _ptr(d_raw2), nf,
                                              first_frame, _ptr(d_acc), _stream(stream)))


def host_register(buf: np.ndarray):
    """fxc_host_register: page-lock a caller-owned numpy buffer in place."""
    check(lib().fxc_host_register(buf.ctypes.data, buf.nbytes))


def host_unregister(buf: np.ndarray):
    check(lib().fxc_host_unregister(buf.ctypes.data))


def sector_noalloc_check(stream=None):
    """fxc_sector_noalloc_check: synchronises `stream` and raises FxcError
    (FXC_ETIMEDOUT, FXC_EDEVICE) when the last allocation-free call on the
    current device reported a kernel error."""
    check(lib().fxc_sector_noalloc_check(_stream(stream)))


def debug_inject_wait_timeout(wait_polls: int = 0, withhold_copies: bool = False):
    """Failure-injection test hook (fxc_debug_inject_wait_timeout): bound the
    correlation kernels' staging waits to `wait_polls` polls and, with
    `withhold_copies`, let them run out with no copy in flight.  (0, False)
    restores normal operation."""
    check(lib().fxc_debug_inject_wait_timeout(wait_polls, int(bool(withhold_copies))))


def probe_exchange(device: int = 0) -> dict:
    """fxc_probe_exchange: ns for one SM to redistribute 8192 complex values
    among 512 threads through shared memory and by warp shuffles."""
    a, b = C.c_double(), C.c_double()
    check(lib().fxc_probe_exchange(device, C.byref(a), C.byref(b)))
    return {"smem_ns": a.value, "shfl_ns": b.value}


def probe_mma_f16(device: int = 0) -> float:
    """fxc_probe_mma_f16: mma.sync m16n8k16 f16 throughput (TFLOP/s)."""
    out = C.c_double()
    check(lib().fxc_probe_mma_f16(device, C.byref(out)))
    return out.value


def probe_fp32_peak(device: int = 0) -> float:
    out = C.c_double()
    check(lib().fxc_probe_fp32_peak(device, C.byref(out)))
    return out.value
