#!/usr/bin/env python
"""Benchmark of the B200 FX-correlation path on the full-rate plain workload:
1024 Msps, 2-bit, FFT 8192, a 10-s scan (10 sectors x 125000 frame pairs),
seeded non-identity 32-bit shuffle, station 1 LSB / station 2 USB with band
centres 16 MHz apart, geometric delay with a 0.5 Hz fringe rate, residual
delay 0.3 samples and residual rate 0.01 Hz, products ACF x2 + XCF.

A step is one pass of the hot path over the whole 10-s scan.  Prints one JSON
line (rank 0).  `--impl reference` times the CPU restatement of the
reference's rayon path (oracle/fxc_oracle.c, OpenMP over all host threads)
on a bounded sample of the same workload instead.

Multi-GPU (torchrun, N ranks): the path does not shard within a scan, so each
rank correlates its own replica scan (weak scaling, no data-path collective);
timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "fx-corr_b200"))

# ---------------------------------------------------------------- workload

N = 8192
FS = 1024e6
BITS = 2
SCAN_S = 10
SECTORS = 10
NF_SECTOR = int(FS / N)  # 125000 frames per 1-s sector
LEVELS = [-3.0, -1.0, 1.0, 3.0]
OBS_MHZ = 8400.0
ROT1_HZ, ROT2_HZ = 0.0, 16e6
RHO = 0.05
METRIC = "Gsample/s (2-bit, FFT 8192)"
WORKLOAD = ("full-rate plain scan: 1024 Msps, 2-bit, FFT 8192, 10 s (10 sectors x 125000 frame "
            "pairs), generic shuffle, ant1 LSB / ant2 USB, 16 MHz band offset, ACFx2+XCF")


def shuffle_internal(seed: int):
    rng = np.random.Generator(np.random.PCG64(seed))
    while True:
        p = [int(v) for v in rng.permutation(32)]
        if p != list(range(32)) and p != [i ^ 1 for i in range(32)]:
            return p


PROD_ACF, PROD_XCF = 1, 2  # product bits (same values in fxc and the oracle)


def scan_fields(band_alignment, fft=N, rot2_hz=ROT2_HZ):
    """Resolve the scan the way run_once does (src/main.rs:1186-1212,
    1317-1328, 1618-1673) for the synthetic schedule above.  Returns the
    fields shared by fxc.ScanConfig and oracle.Scan; `band_alignment` is
    either's restatement of compute_band_alignment (src/main.rs:360-372).
    `fft` other than 8192: the same schedule at another FFT length (the
    --fft-sweep mode); `rot2_hz`: another band offset of station 2."""
    ROT2_HZ = rot2_hz
    bw = FS / 2e6
    c1 = OBS_MHZ + ROT1_HZ / 1e6 + 0.5 * bw
    c2 = OBS_MHZ + ROT2_HZ / 1e6 + 0.5 * bw
    band = band_alignment(fft, FS, c1, c2, bw, bw)
    grid = 0 if abs(ROT1_HZ) <= abs(ROT2_HZ) else 1
    df = FS / fft
    rot_residual = (ROT1_HZ - ROT2_HZ) - band[0] * df
    rate_user = 0.01  # --resrate
    extra_rate = (-rot_residual + rate_user) / (OBS_MHZ * 1e6)
    gr = -0.5 / (OBS_MHZ * 1e6)  # geometric rate giving a 0.5 Hz fringe at obs freq
    gd0 = 2.1e-7
    table = gd0 + gr * np.arange(SCAN_S + 1, dtype=np.float64)
    user = 0.3  # --resdelay
    net_d0 = gd0 + user / FS
    init = int(round(net_d0 * FS))
    start2 = max(init, 0)
    spw = 32 // BITS
    d_seek = ((start2 // spw) * spw - 0) / FS
    delay = dict(time_offset_s=0.0, delay_user_samples=user, extra_delay_rate_sps=extra_rate,
                 d_seek=d_seek, lo1_hz=(OBS_MHZ + ROT1_HZ / 1e6) * 1e6,
                 lo2_hz=(OBS_MHZ + ROT2_HZ / 1e6) * 1e6)
    return dict(fft=fft, fs=FS, bits1=BITS, bits2=BITS, levels1=LEVELS, levels2=LEVELS,
                shuffle1=shuffle_internal(101), shuffle2=shuffle_internal(102),
                lsb1=True, lsb2=False, band=tuple(band), grid=grid,
                products=PROD_ACF | PROD_XCF, delay=delay, geom_table=table)


def scan_config(fxc):
    return fxc.ScanConfig(**scan_fields(fxc.band_alignment))


def import_oracle():
    """The checker and CPU restatement under oracle/ (the bench's CPU legs
    only)."""
    p = str(ROOT / "oracle")
    if p not in sys.path:
        sys.path.insert(0, p)
    import oracle

    return oracle


def oracle_scan():
    """The same scan for the CPU restatement, resolved with the oracle's own
    band alignment (no product code involved)."""
    oracle = import_oracle()
    return oracle.Scan(**scan_fields(oracle.c_band_alignment))


def gen_station_pair_gpu(torch, nsamp, seed, cfg, lag=7):
    """Seeded quantised Gaussian streams (+-0.98 sigma thresholds, levels
    +-1/+-3) sharing a common component at rho=0.05, station 2 lagging by
    `lag` samples, packed into the .raw layout each station's decoder reads."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    chunk = 1 << 26
    a, b = math.sqrt(RHO), math.sqrt(1 - RHO)
    outs = [torch.empty(nsamp * BITS // 8, dtype=torch.uint8, device="cuda") for _ in range(2)]
    prev_tail = torch.randn(lag, device="cuda", generator=g)
    for s0 in range(0, nsamp, chunk):
        m = min(chunk, nsamp - s0)
        c = torch.randn(m, device="cuda", generator=g)
        c_lag = torch.cat([prev_tail, c])[:m]
        prev_tail = c[m - lag:]
        xs = (a * c + b * torch.randn(m, device="cuda", generator=g),
              a * c_lag + b * torch.randn(m, device="cuda", generator=g))
        for st, (x, lsb, sh) in enumerate(zip(xs, (cfg.lsb1, cfg.lsb2),
                                              (cfg.shuffle1, cfg.shuffle2))):
            if lsb:
                x = x.view(-1, 2)
                x[:, 1].neg_()
                x = x.view(-1)
            code = ((x >= -0.98).int() + (x >= 0).int() + (x >= 0.98).int()).view(-1, 16)
            shifts = torch.arange(16, device="cuda", dtype=torch.int64) * 2
            w = (code.long() << shifts).sum(1)
            out = torch.zeros_like(w)
            for pos in range(32):
                out |= ((w >> pos) & 1) << sh[pos]
            outs[st][s0 * BITS // 8:(s0 + m) * BITS // 8] = (
                out.to(torch.int32).view(torch.uint8))
    return outs


# ------------------------------------------------------------------- clocks

class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None
        self.lines = []

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        self.lines += [ln for ln in out.splitlines() if ln.strip()]
        return self.summary()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------- peaks

def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic_per_frame_pair():
    """DRAM bytes per frame pair of the correlation kernel from the committed
    ncu summary (profiles/corr_fold_kernel_n8192.txt), or None."""
    f = ROOT / "profiles" / "corr_fold_kernel_n8192.txt"
    if not f.exists():
        return None
    for ln in f.read_text().splitlines():
        if ln.strip().startswith("dram_bytes_per_frame_pair:"):
            try:
                return float(ln.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def flops_per_station_sample(n):
    return 2.5 * math.log2(n) + 6.5


# -------------------------------------------------------------- CPU legs

def replica_throughput(dist, samples, ms, device):
    """Whole-job throughput of independent replicas (the path shards by scan
    or sector with no data-path collective): every rank's samples over the
    slowest rank's time.  Returns (Gsample/s, slowest ms); dist None = one
    process."""
    if dist is None:
        return samples / (ms * 1e-3) / 1e9, ms
    import torch

    t_ms = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    t_n = torch.tensor([float(samples)], dtype=torch.float64, device=device)
    dist.all_reduce(t_ms, op=dist.ReduceOp.MAX)
    dist.all_reduce(t_n, op=dist.ReduceOp.SUM)
    ms, samples = float(t_ms.item()), float(t_n.item())
    return samples / (ms * 1e-3) / 1e9, ms


def reference_line(steps, warmup, world, sectors=SECTORS, nfs=NF_SECTOR, threads=None):
    """The reference arm: the CPU restatement of the reference's rayon path
    (oracle/fxc_oracle.c, OpenMP over all host threads) on the full workload,
    every step correlating all `sectors` x `nfs` frame pairs of the scan.
    Imports the oracle only, never the product package.  Each sector
    correlates the same seeded 1-s input bytes (generated once by the
    oracle's C generator) with its own delay model (frames i*nfs onwards);
    the restatement's cost does not depend on the sample values."""
    oracle = import_oracle()
    oracle.build()
    scan = oracle_scan()
    threads = threads or os.cpu_count() or 1
    r1, r2 = oracle.synth_packed_pair(nfs * N, 1000, BITS, LEVELS, scan.shuffle1, scan.lsb1,
                                      scan.shuffle2, scan.lsb2, rho=RHO, lag=7, nthreads=threads)

    def step():
        for i in range(sectors):
            out = oracle.c_sector_corr(scan, r1, r2, nfs, i * nfs, threads)
            if out["failed"]:
                raise RuntimeError("restatement reported failed frames")

    for _ in range(warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    dt = (time.perf_counter() - t0) / steps
    value = 2 * sectors * nfs * N / dt / 1e9
    full = sectors == SECTORS and nfs == NF_SECTOR
    sample = (f"the whole scan per step: {sectors} sectors x {nfs} frame pairs (each sector the "
              f"same seeded input bytes with its own delay model)")
    return {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "Gsample/s", "n_gpus": world, "steps": steps, "warmup": warmup,
        "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded quantised Gaussian, "
        "rho=0.05, oracle C generator)",
        "config": {"workload": WORKLOAD if full else
                   f"reduced case ({sectors} x {nfs} frame pairs) of: {WORKLOAD}",
                   "fft": N, "fs_hz": FS, "bits": BITS, "scan_s": SCAN_S,
                   "sectors": sectors, "frames_per_sector": nfs},
        "cpu_baseline": {"value": value, "unit": "Gsample/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "Gsample/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def run_reference(args, rank, world):
    """--impl reference: rank 0 times the CPU restatement on this box's host
    cores; the other ranks exit without work."""
    if rank != 0:
        return 0
    line = reference_line(args.steps, args.warmup, world, args.sectors, args.frames_per_sector)
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ main

def cpu_parity_leg(torch, scan, sec1, sec2, accs, nfs, slice_frames=1000):
    """The CPU restatement of the reference path (oracle/fxc_oracle.c,
    OpenMP over all host threads) on every sector of the measured scan, the
    same bytes the GPU correlated: its time is the cpu_baseline, and its
    accumulators check the GPU's (accs[i], left by the timed steps) at full
    size.  On the first `slice_frames` frames of each sector the GPU, the
    restatement and the FP64 oracle are compared as well, stating the
    restatement's own drift from FP64 beside the GPU's error."""
    oracle = import_oracle()
    sys.path.insert(0, str(ROOT / "tests"))
    from _cases import spectral_errors, xcf_drift_bound, xcf_floor

    oracle.build()
    cfg_o = oracle_scan()
    threads = os.cpu_count() or 1
    h = cfg_o.h
    sb, a1s, a1e, a2s = cfg_o.band
    bound = xcf_drift_bound(a1e - a1s)
    worst = {}

    def upd(key, errs, names):
        d = worst.setdefault(key, {})
        for nm, v in zip(names, errs):
            d[nm] = max(d.get(nm, 0.0), float(v))

    def split(a):
        return dict(acf11=a[:h], acf22=a[h:2 * h], xcf=a[2 * h:4 * h].view(np.complex128))

    names = ("rel_amp", "phase_rad", "abs_over_peak")
    spent, frames = 0.0, 0
    acc_s = torch.empty(5 * h, dtype=torch.float64, device="cuda")
    bpf = cfg_o.bpf(BITS)
    for i in range(len(sec1)):
        r1, r2 = sec1[i].cpu().numpy(), sec2[i].cpu().numpy()
        t0 = time.perf_counter()
        c = oracle.c_sector_corr(cfg_o, r1, r2, nfs, i * nfs, threads)
        spent += time.perf_counter() - t0
        frames += nfs
        g = split(accs[i].cpu().numpy())
        for k in ("acf11", "acf22"):
            upd("gpu_vs_port_" + k, spectral_errors(g[k], c[k]), names)
        upd("gpu_vs_port_xcf", spectral_errors(g["xcf"], c["xcf"], xcf_floor(c, nfs)), names)
        # slice against FP64
        m = min(slice_frames, nfs)
        scan.run_device(sec1[i][:m * bpf], sec2[i][:m * bpf], m, i * nfs, acc_s)
        gs = split(acc_s.cpu().numpy())
        f = oracle.fp64_sector_corr(cfg_o, r1[:m * bpf], r2[:m * bpf], m, i * nfs)
        cs = oracle.c_sector_corr(cfg_o, r1[:m * bpf], r2[:m * bpf], m, i * nfs, threads)
        fl = xcf_floor(f, m)
        for who, x in (("gpu", gs), ("port", cs)):
            for k in ("acf11", "acf22"):
                upd(f"{who}_vs_fp64_{k}", spectral_errors(x[k], f[k]), names)
            upd(f"{who}_vs_fp64_xcf", spectral_errors(x["xcf"], f["xcf"], fl), names)
    scan.check()
    tol_amp, tol_ph = 1e-5, 1e-4
    ok_fp64 = all(worst[f"gpu_vs_fp64_{k}"]["rel_amp"] <= tol_amp and
                  worst[f"gpu_vs_fp64_{k}"]["phase_rad"] <= tol_ph and
                  worst[f"gpu_vs_fp64_{k}"]["abs_over_peak"] <= tol_amp
                  for k in ("acf11", "acf22", "xcf"))
    ok_port = all(worst[f"gpu_vs_port_{k}"]["rel_amp"] <= tol_amp for k in ("acf11", "acf22")) \
        and worst["gpu_vs_port_xcf"]["rel_amp"] <= bound["rel_amp"] \
        and worst["gpu_vs_port_xcf"]["phase_rad"] <= bound["phase_rad"]
    parity = {
        "full_size": {"against": "C restatement of the reference path, same bytes",
                      "sectors": len(sec1), "frame_pairs_compared": frames,
                      **{k[len("gpu_vs_port_"):]: v for k, v in worst.items()
                         if k.startswith("gpu_vs_port_")},
                      "tolerance": {"acf_rel_amp": tol_amp, "xcf": bound,
                                    "xcf_note": "the restatement's f32 phase-ramp recurrence "
                                                "drift (ov * 2^-23) plus the GPU's FP64 "
                                                "tolerance"},
                      "pass": bool(ok_port)},
        "fp64_slices": {"frame_pairs_compared": len(sec1) * min(slice_frames, nfs),
                        "slices": f"first {min(slice_frames, nfs)} frame pairs of each sector",
                        "gpu": {k[len("gpu_vs_fp64_"):]: v for k, v in worst.items()
                                if k.startswith("gpu_vs_fp64_")},
                        "reference_restatement": {k[len("port_vs_fp64_"):]: v
                                                  for k, v in worst.items()
                                                  if k.startswith("port_vs_fp64_")},
                        "tolerance": {"rel_amp": tol_amp, "phase_rad": tol_ph},
                        "pass": bool(ok_fp64)},
        "metrics": "per-bin relative amplitude against max(|ref|, floor), phase on bins at or "
                   "above the floor, largest complex error over the peak (tests/_cases.py)",
    }
    cpu = {"value": 2 * frames * N / spent / 1e9, "unit": "Gsample/s", "cores": threads,
           "kind": "port",
           "sample": f"the whole scan, {len(sec1)} sectors x {nfs} frame pairs ({spent:.1f} s of "
                     f"CPU work, C restatement, OpenMP over all host threads)"}
    # the reference's own default pool: logical cores - 2 (src/main.rs:920-924)
    thr_d = max(1, threads - 2)
    r1, r2 = sec1[0].cpu().numpy(), sec2[0].cpu().numpy()
    t0 = time.perf_counter()
    oracle.c_sector_corr(cfg_o, r1, r2, nfs, 0, thr_d)
    dt = time.perf_counter() - t0
    cpu["at_reference_default_threads"] = {
        "value": 2 * nfs * N / dt / 1e9, "threads": thr_d,
        "sample": f"sector 0, {nfs} frame pairs ({dt:.1f} s of CPU work)"}
    return cpu, parity


def serve_jobs(n_jobs, load, seed=5150):
    """Long jobs: seeded Poisson stream of 0.1-5 s chunks at 256-1024 Msps,
    2-bit, FFT 1024-16384, random station delays and rates, dumps every
    second; arrivals at `load` x real time (data seconds offered per second)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    mean_dur = 2.55
    t = 0.0
    jobs = []
    for k in range(n_jobs):
        t += float(rng.exponential(mean_dur / load))
        dur = float(rng.uniform(0.1, 5.0))
        fs = float(rng.choice([256e6, 512e6, 1024e6]))
        fft = int(rng.choice([1024, 2048, 4096, 8192, 16384]))
        nf = max(1, int(round(dur * fs / fft)))
        delay = dict(frame_dt=fft / fs, fs=fs, net_d1_base=float(rng.uniform(-2e-6, 2e-6)),
                     total_rate1_base=float(rng.uniform(-1e-6, 1e-6)),
                     net_d2_base=float(rng.uniform(-2e-6, 2e-6)), lo1_hz=8.4e9, lo2_hz=8.4e9)
        jobs.append(dict(arrival=t, dur=dur, fs=fs, fft=fft, nf=nf,
                         sector_frames=max(1, int(round(fs / fft))), delay=delay, seed=k))
    return jobs


def short_jobs(n_jobs, rate, seed=6262):
    """Short jobs: seeded Poisson stream at `rate` jobs/s of 1-16 ms chunks
    (125-2000 frame pairs) at 1024 Msps, 2-bit, FFT 8192, random station
    delays and rates, one dump per job."""
    rng = np.random.Generator(np.random.PCG64(seed))
    fs, fft = 1024e6, 8192
    t = 0.0
    jobs = []
    for k in range(n_jobs):
        t += float(rng.exponential(1.0 / rate))
        dur = float(rng.uniform(1e-3, 16e-3))
        nf = max(1, int(round(dur * fs / fft)))
        delay = dict(frame_dt=fft / fs, fs=fs, net_d1_base=float(rng.uniform(-2e-6, 2e-6)),
                     total_rate1_base=float(rng.uniform(-1e-6, 1e-6)),
                     net_d2_base=float(rng.uniform(-2e-6, 2e-6)), lo1_hz=8.4e9, lo2_hz=8.4e9)
        jobs.append(dict(arrival=t, dur=dur, fs=fs, fft=fft, nf=nf, sector_frames=0, delay=delay,
                         seed=k))
    return jobs


def batch_leg(fxc, torch, eng, n_sectors=64, calls=20, warm=3, seed=8383):
    """Device-resident batched throughput: one fxc_batch call = one sector
    each of n_sectors distinct short 2-bit FFT-8192 scans (125-2000 frame
    pairs, random delays), replayed from a CUDA graph with the autotuned
    shape; CUDA events around each call on the calling stream."""
    jobs = short_jobs(n_sectors, rate=1.0, seed=seed)
    scans, r1, r2, accs, nfs = [], [], [], [], []
    tot = sum(j["nf"] for j in jobs) * (N * BITS // 8)
    g = torch.Generator(device="cuda").manual_seed(seed)
    d = torch.randint(0, 256, (2, tot), dtype=torch.uint8, device="cuda", generator=g)
    off = 0
    for j in jobs:
        c = fxc.ScanConfig(fft=j["fft"], fs=j["fs"], bits1=2, bits2=2,
                           levels1=[-3.0, -1.0, 1.0, 3.0], levels2=[-3.0, -1.0, 1.0, 3.0],
                           shuffle1=shuffle_internal(101), shuffle2=shuffle_internal(102),
                           products=fxc.PROD_ACF | fxc.PROD_XCF, delay=j["delay"])
        scans.append(eng.open_scan(c))
        n = j["nf"] * c.bpf(2)
        r1.append(d[0, off:off + n])
        r2.append(d[1, off:off + n])
        off += n
        accs.append(torch.empty(5 * c.h, dtype=torch.float64, device="cuda"))
        nfs.append(j["nf"])
    b = fxc.Batch(eng, use_graphs=True, autotune=True)
    st = torch.cuda.current_stream()
    firsts = [0] * n_sectors
    for _ in range(warm):
        b.run_device(scans, r1, r2, nfs, firsts, accs, stream=st)
    torch.cuda.synchronize()
    l0 = b.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(calls):
        b.run_device(scans, r1, r2, nfs, firsts, accs, stream=st)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / calls
    for s in scans:
        s.check()
    samples = 2.0 * N * sum(nfs)
    out = {"gsample_s": samples / (ms * 1e-3) / 1e9, "ms_per_call": ms,
           "sectors_per_call": n_sectors, "frame_pairs_per_call": int(sum(nfs)),
           "kernels_per_call": (b.launches() - l0) / calls, "shape_fft8192": b.shape(N),
           "input_bytes_per_call": 2 * tot,
           "path": "fxc_batch_run_device (CUDA graph replay: frame records, one persistent "
                   "corr_fold_batch_kernel, one reduction), device-resident inputs"}
    b.close()
    for s in scans:
        s.close()
    del d
    return out


def batch_mixed_leg(fxc, torch, eng, n_scans=64, calls=10, warm=3, seed=9494):
    """The batched multi-scan schedule's shape: one fxc_batch call = one
    sector each of n_scans scans with FFT lengths {1024, 4096, 16384}, bit
    depths {1, 2, 4} (both stations) and, alternately, the correlation
    (ACF x2 + XCF) or the phased (power + .raw) products; uneven sectors of
    0.05-0.3 s at 512 Msps with random delays; CUDA graphs and the autotuner
    on; CUDA events around each call.  Device-resident random .raw bytes."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ffts, bitss = (1024, 4096, 16384), (1, 2, 4)
    fs = 512e6
    specs = []
    for k in range(n_scans):
        fft = ffts[k % 3]
        bits = bitss[(k // 3) % 3]
        phased = (k // 9) % 2 == 1
        nf = max(1, int(rng.uniform(0.05, 0.3) * fs / fft))
        delay = dict(net_d1_base=float(rng.uniform(-3e-6, 3e-6)),
                     total_rate1_base=float(rng.uniform(-2e-6, 2e-6)), lo1_hz=8.4e9, lo2_hz=8.4e9)
        specs.append((fft, bits, phased, nf, delay))
    levels = {1: [-1.0, 1.0], 2: [-3.0, -1.0, 1.0, 3.0],
              4: [float(v) for v in np.arange(-7.5, 8.0, 1.0)]}
    scans, r1, r2, accs, nfs, raws = [], [], [], [], [], []
    tot = sum(nf * fft * bits // 8 for fft, bits, _, nf, _ in specs)
    g = torch.Generator(device="cuda").manual_seed(seed)
    d = torch.randint(0, 256, (2, tot), dtype=torch.uint8, device="cuda", generator=g)
    off = 0
    for fft, bits, phased, nf, delay in specs:
        c = fxc.ScanConfig(fft=fft, fs=fs, bits1=bits, bits2=bits, levels1=levels[bits],
                           levels2=levels[bits], shuffle1=shuffle_internal(101),
                           shuffle2=shuffle_internal(102),
                           products=(fxc.PROD_PHASED | fxc.PROD_RAW) if phased
                           else (fxc.PROD_ACF | fxc.PROD_XCF), delay=delay)
        scans.append(eng.open_scan(c))
        n = nf * c.bpf(bits)
        r1.append(d[0, off:off + n])
        r2.append(d[1, off:off + n])
        off += n
        accs.append(torch.empty(5 * c.h, dtype=torch.float64, device="cuda"))
        raws.append(torch.empty(n, dtype=torch.uint8, device="cuda") if phased else None)
        nfs.append(nf)
    b = fxc.Batch(eng, use_graphs=True, autotune=True)
    st = torch.cuda.current_stream()
    firsts = [0] * n_scans
    for _ in range(warm):
        b.run_device_raw(scans, r1, r2, nfs, firsts, accs, raws, stream=st)
    torch.cuda.synchronize()
    l0 = b.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(calls):
        b.run_device_raw(scans, r1, r2, nfs, firsts, accs, raws, stream=st)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / calls
    for s in scans:
        s.check()
    samples = sum(2.0 * fft * nf for fft, _, _, nf, _ in specs)
    # every sector of this mix has a batch group (none runs through its scan's
    # own kernels inside the call)
    per_scan = 0
    out = {"gsample_s": samples / (ms * 1e-3) / 1e9, "ms_per_call": ms, "scans": n_scans,
           "frame_pairs_per_call": int(sum(nfs)), "input_bytes_per_call": 2 * tot,
           "kernels_per_call": (b.launches() - l0) / calls,
           "sectors_in_persistent_kernels": n_scans - per_scan,
           "sectors_through_per_scan_kernels": per_scan,
           "mix": "FFT {1024, 4096, 16384} x bits {1, 2, 4} x {ACF+XCF, phased power + .raw}, "
                  "0.05-0.3 s sectors at 512 Msps, random delays",
           "path": "fxc_batch_run_device_raw (CUDA graph replay, autotuned), device-resident"}
    b.close()
    for s in scans:
        s.close()
    del d
    return out


def serve_leg(fxc, torch, eng, jobs, slots, batch, plain_jobs=None, label="", mix=""):
    """Served (fxc_server, continuous batching) vs plain (one job at a time:
    scan open, per sector a synchronous H2D + kernels + dump, scan close) on
    the same job stream, at the offered arrival times and saturated (all jobs
    queued at once).  plain_jobs: the plain path runs only the first jobs of
    the stream (its throughput per job is that of a sequential loop)."""
    import threading

    cfgs = []
    for j in jobs:
        c = fxc.ScanConfig(fft=j["fft"], fs=j["fs"], bits1=2, bits2=2,
                           levels1=[-3.0, -1.0, 1.0, 3.0], levels2=[-3.0, -1.0, 1.0, 3.0],
                           shuffle1=shuffle_internal(101), shuffle2=shuffle_internal(102),
                           products=fxc.PROD_ACF | fxc.PROD_XCF, delay=j["delay"])
        cfgs.append(c)
    need = max(j["nf"] * j["fft"] * 2 // 8 for j in jobs)
    pool = []
    for st in range(2):
        g = torch.Generator(device="cuda").manual_seed(77 + st)
        d = torch.randint(0, 256, (need,), dtype=torch.uint8, device="cuda", generator=g)
        hbuf = torch.empty(need, dtype=torch.uint8, pin_memory=True)
        hbuf.copy_(d)
        pool.append(hbuf)
        del d
    torch.cuda.synchronize()
    p1, p2 = pool[0].numpy(), pool[1].numpy()
    samples = [2 * j["nf"] * j["fft"] for j in jobs]
    np_jobs = len(jobs) if plain_jobs is None else min(plain_jobs, len(jobs))

    def plain_job(j, c):
        # the plain single-job path: open a scan, then per sector a synchronous
        # H2D from pinned memory, the kernels and the dump, then close
        s = eng.open_scan(c)
        b = c.bpf(2)
        sf = j["sector_frames"] or j["nf"]
        for f0 in range(0, j["nf"], sf):
            n = min(sf, j["nf"] - f0)
            s.wait(s.submit(p1[f0 * b:(f0 + n) * b], p2[f0 * b:(f0 + n) * b], n, f0))
        s.close()

    def run_plain(paced):
        lat = []
        t0 = time.perf_counter()
        for j, c in list(zip(jobs, cfgs))[:np_jobs]:
            arr = t0 + (j["arrival"] if paced else 0.0)
            now = time.perf_counter()
            if now < arr:
                time.sleep(arr - now)
            plain_job(j, c)
            lat.append(time.perf_counter() - arr)
        return lat, time.perf_counter() - t0

    sv = fxc.Server(eng, slots=slots, batch=batch)  # long-lived: slots keep their device state

    # the client's job descriptors and output blocks, built once: the timed
    # loops are one C-ABI call per submission and per wait
    import ctypes as C

    L = fxc.lib()
    cfg_cs = [c.to_c() for c in cfgs]
    prepared = []
    for k, (j, c) in enumerate(zip(jobs, cfgs)):
        sf = j["sector_frames"] or max(j["nf"], 1)
        out = np.zeros(((j["nf"] + sf - 1) // sf, 5 * c.h))
        jc = fxc.JobC(C.addressof(cfg_cs[k]), p1.ctypes.data, p2.ctypes.data, j["nf"], 0,
                      j["sector_frames"], out.ctypes.data, None)
        prepared.append((jc, out))

    def run_served(paced, server=None, count=None):
        server = server or sv
        n = len(jobs) if count is None else count
        ids = [C.c_uint64() for _ in range(n)]
        stats = [fxc.JobStats() for _ in range(n)]
        ready = [threading.Event() for _ in range(n)]
        err = []
        t0 = time.perf_counter()

        def submitter():
            for k in range(n):
                if paced:
                    dt = t0 + jobs[k]["arrival"] - time.perf_counter()
                    if dt > 0:
                        time.sleep(dt)
                rc = L.fxc_server_submit(server.h, C.byref(prepared[k][0]), C.byref(ids[k]))
                if rc != 0:
                    err.append((k, rc, L.fxc_last_error().decode()))
                ready[k].set()

        th = threading.Thread(target=submitter)
        th.start()
        for k in range(n):  # waits run beside the submissions
            ready[k].wait()
            if not err:
                rc = L.fxc_server_wait(server.h, ids[k].value, -1, C.byref(stats[k]))
                if rc != 0:
                    err.append((k, rc, L.fxc_last_error().decode()))
        th.join()
        if err:
            raise RuntimeError(f"served job failed: {err[0]}")
        # the server's own clock: first submission to last completion
        wall = (max(x.t_done_ns for x in stats) - min(x.t_submit_ns for x in stats)) * 1e-9
        return [(x.t_done_ns - x.t_submit_ns) * 1e-9 for x in stats], wall

    try:
        # warm both paths (module load; the server's slots grow to the job mix
        # and the batch autotuner runs at its first batch of each FFT length)
        plain_job(jobs[0], cfgs[0])
        run_served(False)
        run_served(False)
        # saturated: every job queued at once, median of three runs each
        p_sat_wall = statistics.median(run_plain(False)[1] for _ in range(3))
        s_sat_wall = statistics.median(run_served(False)[1] for _ in range(3))
        s_lat, s_wall = run_served(True)
        p_lat, p_wall = run_plain(True)
    finally:
        sv.close()
    # the second plain baseline: one job at a time through one long-lived scan
    # that is rebound to each job (a one-slot server without batching: no
    # per-job allocation, the job loop runs in the server's C++ worker)
    pp = fxc.Server(eng, slots=1, batch=False)
    try:
        run_served(False, pp, np_jobs)
        q_sat_wall = statistics.median(run_served(False, pp, np_jobs)[1] for _ in range(3))
        q_lat, q_wall = run_served(True, pp, np_jobs)
    finally:
        pp.close()
    tot = float(sum(samples))
    tot_plain = float(sum(samples[:np_jobs]))

    def pct(v, q):
        return float(np.percentile(np.asarray(v) * 1e3, q))

    s_jps, p_jps = len(jobs) / s_sat_wall, np_jobs / p_sat_wall
    q_jps = np_jobs / q_sat_wall
    return {
        "workload": label, "jobs": len(jobs), "plain_jobs": np_jobs, "slots": slots,
        "batched": bool(batch), "job_mix": mix,
        "data_s_per_job_mean": float(np.mean([j["dur"] for j in jobs])),
        "served": {"p50_ms": pct(s_lat, 50), "p99_ms": pct(s_lat, 99),
                   "gsample_s": tot / s_wall / 1e9,
                   "saturated_jobs_per_s": s_jps,
                   "saturated_gsample_s": tot / s_sat_wall / 1e9},
        "plain": {"p50_ms": pct(p_lat, 50), "p99_ms": pct(p_lat, 99),
                  "gsample_s": tot_plain / p_wall / 1e9,
                  "saturated_jobs_per_s": p_jps,
                  "saturated_gsample_s": tot_plain / p_sat_wall / 1e9,
                  "path": "per job: fxc_scan_open, per-sector synchronous fxc_sector_submit/wait, "
                          "fxc_scan_close (Python loop)"},
        "plain_persistent": {"p50_ms": pct(q_lat, 50), "p99_ms": pct(q_lat, 99),
                             "gsample_s": tot_plain / q_wall / 1e9,
                             "saturated_jobs_per_s": q_jps,
                             "saturated_gsample_s": tot_plain / q_sat_wall / 1e9,
                             "path": "one long-lived scan rebound to each job in turn (one-slot "
                                     "server, no batching): no per-job allocation, job loop in "
                                     "C++"},
        "saturated_job_throughput_ratio": s_jps / p_jps,
        "saturated_job_throughput_ratio_vs_persistent": s_jps / q_jps,
        "saturated_runs": "median of 3 per path",
        "path": "fxc_server_submit/fxc_server_wait%s" % (
            " (batched: fxc_batch_run_device in CUDA graphs, autotuned)" if batch else ""),
    }


def fft_sweep(args):
    """Device-resident throughput of the correlation and phased (.raw)
    products by FFT length: the full-rate scan's schedule (1024 Msps, 2-bit,
    generic shuffle, LSB/USB, 16 MHz band offset) at each length, one sector
    of --sweep-samples samples per station per call, CUDA events on the
    calling stream over --steps calls after --warmup.  --sweep-bits other than
    2: both stations at that bit depth (odd-integer levels) with random .raw
    bytes.  --sweep-offset-mhz: station 2's band offset (16.0625 MHz gives an
    odd band shift at FFT 16384).  One JSON line; not the benchmark line."""
    import torch

    import fxc

    torch.cuda.set_device(0)
    eng = fxc.Engine(0)
    stream = torch.cuda.Stream()
    bits = args.sweep_bits
    out = {"mode": "fft-sweep", "unit": f"Gsample/s (device-resident, {bits}-bit)",
           "samples_per_station_per_call": args.sweep_samples, "calls": args.steps,
           "band_offset_mhz": args.sweep_offset_mhz}
    for fft in [int(v) for v in args.sweep_ffts.split(",")]:
        for prod in args.sweep_products.split(","):
            fields = scan_fields(fxc.band_alignment, fft=fft, rot2_hz=args.sweep_offset_mhz * 1e6)
            if bits != BITS:
                lv = [float(v) for v in range(1 - (1 << bits), 1 << bits, 2)]
                fields.update(bits1=bits, bits2=bits, levels1=lv, levels2=lv)
            if prod == "phased":
                fields["products"] = fxc.PROD_PHASED | fxc.PROD_RAW
            cfg = fxc.ScanConfig(**fields)
            scan = eng.open_scan(cfg)
            nf = args.sweep_samples // fft
            if bits == BITS:
                d1, d2 = gen_station_pair_gpu(torch, nf * fft, seed=fft, cfg=cfg)
            else:
                g = torch.Generator(device="cuda").manual_seed(fft)
                d1, d2 = (torch.randint(0, 256, (nf * cfg.bpf(bits),), dtype=torch.uint8,
                                        device="cuda", generator=g) for _ in range(2))
            acc = torch.empty(5 * cfg.h, dtype=torch.float64, device="cuda")
            raw = (torch.empty(nf * cfg.bpf(cfg.bits_out), dtype=torch.uint8, device="cuda")
                   if prod == "phased" else None)

            def call():
                scan.run_device(d1, d2, nf, 0, acc, d_raw_out=raw, stream=stream)

            for _ in range(args.warmup):
                call()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                call()
            e1.record(stream)
            torch.cuda.synchronize()
            scan.check()
            ms = e0.elapsed_time(e1) / args.steps
            out[f"{prod}_{fft}"] = round(2 * nf * fft / (ms * 1e-3) / 1e9, 1)
            scan.close()
            del d1, d2, raw
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fxc", choices=["fxc", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer e2e leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-vs-plain leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-sectors leg")
    ap.add_argument("--serve-jobs", type=int, default=20)
    ap.add_argument("--serve-short-jobs", type=int, default=2000)
    ap.add_argument("--sectors", type=int, default=SECTORS,
                    help="sectors per step (profiling cases only; the workload is 10)")
    ap.add_argument("--frames-per-sector", type=int, default=NF_SECTOR,
                    help="frame pairs per sector (profiling cases only; the workload is 125000)")
    ap.add_argument("--fft-sweep", action="store_true",
                    help="print device-resident throughput by FFT length instead of the "
                         "benchmark line")
    ap.add_argument("--sweep-ffts", default="1024,2048,4096,8192,16384,32768,65536")
    ap.add_argument("--sweep-products", default="corr,phased")
    ap.add_argument("--sweep-bits", type=int, default=2, choices=(1, 2, 4, 8),
                    help="--fft-sweep: both stations' bit depth")
    ap.add_argument("--sweep-samples", type=int, default=1 << 29,
                    help="samples per station per call in --fft-sweep")
    ap.add_argument("--sweep-offset-mhz", type=float, default=ROT2_HZ / 1e6,
                    help="station 2's band offset in --fft-sweep")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.fft_sweep:
        return fft_sweep(args)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch

    import fxc

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    cfg = scan_config(fxc)
    eng = fxc.Engine(local, max_inflight=3)
    scan = eng.open_scan(cfg)
    stream = torch.cuda.Stream()

    # ---- inputs resident in HBM: 10 sectors x 2 stations x 256 MB
    SECTORS_, NFS = args.sectors, args.frames_per_sector
    full = SECTORS_ == SECTORS and NFS == NF_SECTOR
    nsamp = SECTORS_ * NFS * N
    d1, d2 = gen_station_pair_gpu(torch, nsamp, seed=1000 + rank, cfg=cfg)
    bpf = N * BITS // 8
    sec_bytes = NFS * bpf
    sec1 = [d1[i * sec_bytes:(i + 1) * sec_bytes] for i in range(SECTORS_)]
    sec2 = [d2[i * sec_bytes:(i + 1) * sec_bytes] for i in range(SECTORS_)]
    h = cfg.h
    accs = [torch.empty(5 * h, dtype=torch.float64, device="cuda") for _ in range(SECTORS_)]

    def step():
        for i in range(SECTORS_):
            scan.run_device(sec1[i], sec2[i], NFS, i * NFS, accs[i], stream=stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    scan.check()
    scan.profile(reset=True)
    scan.set_profiling(True)

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    kern_ms, kern_launches, all_launches = scan.profile(reset=True)
    scan.set_profiling(False)
    scan.check()
    samples_per_step = 2 * SECTORS_ * NFS * N
    value, ms = replica_throughput(dist, samples_per_step, ms, "cuda")

    # ---- end to end through the host-buffer C ABI (pinned host inputs)
    e2e = None
    if not args.no_e2e:
        h1 = [s.cpu().pin_memory() for s in sec1]
        h2 = [s.cpu().pin_memory() for s in sec2]
        n1 = [t.numpy() for t in h1]
        n2 = [t.numpy() for t in h2]

        def e2e_run(steps):
            # a streaming correlator keeps up to 3 sectors in flight across step
            # boundaries; every step's 10 sector results are read back
            ids = []
            res = []
            for _ in range(steps):
                for i in range(SECTORS_):
                    if len(ids) == 3:
                        res.append(scan.wait(ids.pop(0)))
                    ids.append(scan.submit(n1[i], n2[i], NFS, i * NFS))
            while ids:
                res.append(scan.wait(ids.pop(0)))
            assert len(res) == steps * SECTORS_
            return res

        e2e_run(1)
        barrier()
        t0 = time.perf_counter()
        e2e_run(args.e2e_steps)
        t1 = time.perf_counter()
        barrier()
        e2e_v, e2e_ms = replica_throughput(dist, samples_per_step, (t1 - t0) * 1e3 / args.e2e_steps,
                                           "cuda")
        e2e = {"value": e2e_v, "unit": "Gsample/s",
               "h2d_bytes_per_step": 2 * SECTORS_ * sec_bytes,
               "d2h_bytes_per_step": SECTORS_ * (5 * h * 8 + 4), "ms_per_step": e2e_ms,
               "path": "fxc_sector_submit/fxc_sector_wait, pinned host buffers, 3 sectors in "
                       "flight across steps"}
    clk = clocks.stop()

    # ---- batched sectors of many short scans, device-resident (rank 0 of N=1)
    batched = batched_mixed = None
    if rank == 0 and world == 1 and not args.no_batch:
        batched = batch_leg(fxc, torch, eng)
        try:
            batched_mixed = batch_mixed_leg(fxc, torch, eng)
        except Exception as e:  # report, keep the rest of the line
            batched_mixed = {"error": str(e)[:300]}

    # ---- serving: continuous batching vs one job at a time (rank 0 of N=1)
    serve = None
    if rank == 0 and world == 1 and not args.no_serve:
        def guarded(fn):
            try:
                return fn()
            except Exception as e:  # report, keep the rest of the line
                return {"error": f"{type(e).__name__}: {e}"}

        serve = {
            # the headline's served vs plain: the long-job stream of the serving
            # workload (0.1-5 s chunks, FFT 1024-16384, 2x real time offered)
            "headline": "long",
            # long sectors saturate the host link from per-slot streams, the
            # server's mode for long scans (batching pays off on short jobs)
            "long": guarded(lambda: serve_leg(
                fxc, torch, eng, serve_jobs(args.serve_jobs, 2.0), slots=4, batch=False,
                label="serving workload: long jobs, mixed FFT",
                mix="Poisson arrivals at 2x real time; 0.1-5 s at 256/512/1024 Msps, 2-bit, "
                    "FFT 1024-16384, random delays/rates, 1-s dumps, pinned host buffers")),
            # a second figure: short 2-bit FFT-8192 jobs, where per-job set-up
            # dominates the plain path
            "short": guarded(lambda: serve_leg(
                fxc, torch, eng, short_jobs(args.serve_short_jobs, rate=4000.0), slots=32,
                batch=True, plain_jobs=200, label="short jobs, FFT 8192",
                mix="Poisson arrivals at 4000 jobs/s; 1-16 ms at 1024 Msps (125-2000 frame "
                    "pairs), 2-bit, FFT 8192, random delays/rates, one dump, pinned host buffers")),
        }

    # ---- roofline of the dominant kernel (correlation kernel, one sector per launch)
    launch_ms = kern_ms / max(1, kern_launches)
    flops_launch = flops_per_station_sample(N) * 2 * NFS * N
    fp32_peak = fxc.probe_fp32_peak(local)
    hbm_peak, peak_kind = measured_peaks()
    bytes_launch = 2 * sec_bytes + 5 * h * 8
    tpf = profile_traffic_per_frame_pair()
    roofline = {
        "bound": "fp32", "achieved": flops_launch / (launch_ms * 1e-3) / 1e12,
        "peak": fp32_peak, "unit": "TFLOP/s",
        "frac": flops_launch / (launch_ms * 1e-3) / 1e12 / fp32_peak,
        "traffic": None if tpf is None else tpf * NFS,
        "kernel": "corr_fold_kernel (FFT 8192)", "launch_ms": launch_ms,
        "algorithmic_flops_per_launch": flops_launch,
        "peak_source": "live FMA probe of this GPU (fxc_probe_fp32_peak)",
        "hbm": {"achieved": bytes_launch / (launch_ms * 1e-3) / 1e9, "peak": hbm_peak,
                "unit": "GB/s", "frac": bytes_launch / (launch_ms * 1e-3) / 1e9 / hbm_peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6650 GB/s",
                "algorithmic_bytes_per_launch": bytes_launch},
    }

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu, parity = cpu_parity_leg(torch, scan, sec1, sec2, accs, NFS)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Gsample/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded quantised Gaussian, rho=0.05, generated on device)",
            "config": {"workload": WORKLOAD if full else
                       f"profiling case ({SECTORS_} x {NFS} frame pairs) of: {WORKLOAD}",
                       "fft": N, "fs_hz": FS, "bits": BITS,
                       "scan_s": SCAN_S, "sectors": SECTORS_, "frames_per_sector": NFS,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2 (512 MB per sector, 5.12 GB per step)"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "parity": parity,
            "e2e": e2e,
            "batched": batched,
            "batched_mixed": batched_mixed,
            "serving": serve,
            "gpu_launches": all_launches,
            "clocks": clk,
            "realtime_factor": value / (2 * FS / 1e9),
        }
        print(json.dumps(line), flush=True)
    scan.close()
    eng.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
