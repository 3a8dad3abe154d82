"""Serving loop (fxc_server_*): continuous batching of uneven correlation
jobs.  Every job's dumps must be the same alone, in a mix of concurrent jobs,
under a tight HBM budget, and through the plain per-sector scan API."""
from __future__ import annotations

import numpy as np
import pytest

from _cases import make_scan, random_raw, to_fxc

pytestmark = pytest.mark.gpu

DELAY = dict(net_d1_base=3.3e-7, total_rate1_base=2.1e-6, lo1_hz=8.4e9, lo2_hz=8.4e9)


def make_jobs(seed, count):
    """Uneven jobs: FFT 1024..16384, 1/2/4-bit, 0..700 frames, various dump
    lengths, LSB and grid choices, per-job delays."""
    rng = np.random.Generator(np.random.PCG64(seed))
    jobs = []
    for k in range(count):
        fft = int(rng.choice([1024, 4096, 8192, 16384]))
        bits = int(rng.choice([1, 2, 4]))
        nf = int(rng.integers(0, 700)) if k else 0
        sf = int(rng.choice([0, 64, 250]))
        sb = int(rng.choice([0, 8, -8]))
        band = (sb, max(0, -sb), fft // 2 - max(0, sb), max(0, sb))
        delay = dict(DELAY, net_d1_base=float(rng.uniform(-2e-6, 2e-6)))
        scan = make_scan(fft=fft, fs=512e6, bits1=bits, bits2=int(rng.choice([1, 2, 4])),
                         shuffle=str(rng.choice(["identity", "generic"])), lsb1=bool(k % 2),
                         lsb2=bool(k % 3 == 0), band=band, grid=int(rng.integers(0, 2)),
                         delay=delay, seed=k)
        r1, r2 = random_raw(scan, nf, seed=100 + k)
        jobs.append(dict(cfg=to_fxc(scan), raw1=r1, raw2=r2, nf=nf,
                         first_frame=int(rng.integers(0, 1000)), sector_frames=sf))
    return jobs


def run(server, jobs):
    ids = [server.submit(j["cfg"], j["raw1"], j["raw2"], j["nf"], j["first_frame"],
                         j["sector_frames"]) for j in jobs]
    return [server.wait(i) for i in ids]


def same(a, b):
    assert len(a) == len(b)
    for da, db in zip(a, b):
        for k in ("acf11", "acf22", "xcf", "phased"):
            assert np.array_equal(da[k], db[k]), k


def test_alone_equals_mix(engine):
    import fxc

    jobs = make_jobs(7, 14)
    sv = fxc.Server(engine, slots=4)
    alone = [run(sv, [j])[0] for j in jobs]
    mixed = run(sv, jobs)
    for (da, sa), (dm, sm) in zip(alone, mixed):
        same(da, dm)
        assert sa["sectors"] == sm["sectors"] == len(da)
    # in the mix, jobs overlapped: some job started before an earlier one finished
    starts = [s["t_start_ns"] for _, s in mixed]
    dones = [s["t_done_ns"] for _, s in mixed]
    assert any(starts[i + 1] < dones[i] for i in range(len(jobs) - 1))
    sv.close()


def test_server_equals_scan_path(engine):
    import fxc

    jobs = make_jobs(11, 4)
    sv = fxc.Server(engine, slots=2)
    got = run(sv, jobs)
    sv.close()
    for j, (dumps, st) in zip(jobs, got):
        cfg, nf = j["cfg"], j["nf"]
        sf = j["sector_frames"] or max(nf, 1)
        s = engine.open_scan(cfg)
        ref = []
        for f0 in range(0, max(nf, 1), sf):
            n = min(sf, nf - f0) if nf else 0
            b1, b2 = cfg.bpf(cfg.bits1), cfg.bpf(cfg.bits2)
            sid = s.submit(j["raw1"][f0 * b1:(f0 + n) * b1], j["raw2"][f0 * b2:(f0 + n) * b2],
                           n, j["first_frame"] + f0)
            ref.append(s.wait(sid))
        s.close()
        same(dumps, ref)


def test_tight_budget_admission():
    """Jobs wait for HBM instead of failing while another job can free it."""
    import fxc

    jobs = make_jobs(3, 8)
    big = fxc.Engine(0)
    sv = fxc.Server(big, slots=4)
    ref = run(sv, jobs)
    sv.close()
    big.close()
    # room for about one FFT-16384 job (two 64 MiB batch buffers) at a time
    small = fxc.Engine(0, hbm_budget_bytes=200 << 20)
    sv = fxc.Server(small, slots=4)
    got = run(sv, jobs)
    for (dr, _), (dg, _) in zip(ref, got):
        same(dr, dg)
    sv.close()
    small.close()


def test_bad_job_is_reported_and_server_continues(engine):
    import fxc

    jobs = make_jobs(5, 3)
    bad = make_scan(fft=8192, fs=512e6, delay=DELAY)
    bad_cfg = to_fxc(bad)
    bad_cfg.fft = 3000
    sv = fxc.Server(engine, slots=2)
    jid = sv.submit(bad_cfg, np.zeros(16, np.uint8), np.zeros(16, np.uint8), 0)
    ok = run(sv, jobs)
    with pytest.raises(fxc.FxcError) as ei:
        sv.wait(jid)
    assert ei.value.status == fxc.EUNSUPPORTED
    assert all(st["status"] == 0 for _, st in ok)
    sv.close()


# ----------------------------------------------------------- batched mode

def close_dumps(a, b, jobs_nf):
    """Batched vs per-scan dumps: FP32 agreement (different partial-sum
    grouping), cross-spectra against their noise floor."""
    from _cases import assert_spectra_close, xcf_floor

    assert len(a) == len(b)
    for da, db in zip(a, b):
        for k in ("acf11", "acf22"):
            if np.any(db[k]):
                assert_spectra_close(da[k], db[k], k)
            else:
                assert not np.any(da[k]), k
        fl = xcf_floor(db, jobs_nf)
        if fl is not None:
            assert_spectra_close(da["xcf"], db["xcf"], "xcf", floor=fl)
        assert np.array_equal(da["phased"], db["phased"])


def test_batched_alone_equals_mix_and_matches_plain(engine):
    import fxc

    jobs = make_jobs(7, 14)
    sv = fxc.Server(engine, slots=8, batch=True)
    alone = [run(sv, [j])[0] for j in jobs]
    mixed = run(sv, jobs)
    for (da, sa), (dm, sm) in zip(alone, mixed):
        same(da, dm)  # the item split depends only on the sector and the tuned shape
        assert sa["sectors"] == sm["sectors"] == len(da)
    sv.close()
    plain = fxc.Server(engine, slots=4)
    ref = run(plain, jobs)
    plain.close()
    for j, (dm, _), (dr, _) in zip(jobs, mixed, ref):
        close_dumps(dm, dr, max(1, min(j["nf"], j["sector_frames"] or j["nf"])))


def test_batched_many_short_jobs(engine):
    """Hundreds of one-sector jobs share batches; each equals its alone run."""
    import fxc

    rng = np.random.Generator(np.random.PCG64(99))
    jobs = []
    for k in range(96):
        fft = int(rng.choice([1024, 8192]))
        scan = make_scan(fft=fft, fs=1024e6, bits1=2, bits2=2, shuffle="generic",
                         band=(0, 0, fft // 2, 0), delay=dict(DELAY, net_d2_base=1e-7 * k), seed=k)
        nf = int(rng.integers(1, 300))
        r1, r2 = random_raw(scan, nf, seed=500 + k)
        jobs.append(dict(cfg=to_fxc(scan), raw1=r1, raw2=r2, nf=nf, first_frame=k,
                         sector_frames=0))
    sv = fxc.Server(engine, slots=32, batch=True)
    mixed = run(sv, jobs)
    for j, (dm, st) in zip(jobs[::12], mixed[::12]):
        alone = run(sv, [j])[0][0]
        same(alone, dm)
        assert st["status"] == 0
    sv.close()


def test_batched_tight_budget(engine):
    """Under a tight HBM budget the batched server still finishes every job
    (a batch that does not fit falls back to the per-scan buffers)."""
    import fxc

    jobs = make_jobs(3, 8)
    plain = fxc.Server(engine, slots=2)
    ref = run(plain, jobs)
    plain.close()
    small = fxc.Engine(0, hbm_budget_bytes=200 << 20)
    sv = fxc.Server(small, slots=4, batch=True)
    got = run(sv, jobs)
    for j, (dr, _), (dg, st) in zip(jobs, ref, got):
        assert st["status"] == 0
        close_dumps(dg, dr, max(1, min(j["nf"], j["sector_frames"] or j["nf"])))
    sv.close()
    small.close()
