"""yi-corr end to end on the plain workloads' configurations, with the scan
derived independently by tests/_runonce.py (a restatement of run_once,
src/main.rs:1063-1673) and correlated by the library on the same bytes:

* FFT 1024 at 32 Msps, stations 100 m apart, source at 12h/+30 deg, clock
  offset 1.5 us and rate 1e-12 s/s, 123.4-sample lag: the geometric table is
  live; the tool's .cor equals the library's numbers bit for bit, is within
  tolerance of FP64, and the XCF phase slope recovers the lag;
* the full-rate plain configuration (1024 Msps, FFT 8192, generic shuffle,
  --sideband "ant1:LSB ant2:USB", <rotation> 16 MHz apart, a baseline giving
  a geometric fringe rate, --resdelay 0.3 --resrate 0.01), two 1-s sectors
  (<length>1.5</length>): bit for bit against the library, within tolerance
  of FP64;
* a read start that is not word aligned (the reference reads from the word
  boundary below and keeps the residual in the delay model,
  src/main.rs:1577-1616) and a station file truncated mid-frame (only whole
  frames of the shorter stream are used, src/main.rs:1276-1304);
* a reader error (a station "file" that is a directory): the tool exits 1
  with the reference's message (src/main.rs:2110-2127, 2196-2210)."""
from __future__ import annotations

import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from _cases import assert_sector_close, spectral_errors, to_fxc, xcf_floor
from _runonce import Station, derive, schedule_xml

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "fx-corr_b200" / "bin"
EPOCH, TAG = "2024/043 15:52:00", "2024043155200"
POS1 = (-3502544.587, 3950966.235, 3566381.192)
IDENT_EXT = list(range(31, -1, -1))
LEVELS2 = [-3.0, -1.0, 1.0, 3.0]


def offset(pos, d):
    return tuple(p + q for p, q in zip(pos, d))


def run_tool(name, *args, cwd=None, ok=True):
    r = subprocess.run([str(BIN / name), *map(str, args)], cwd=cwd, capture_output=True,
                       text=True, timeout=900)
    if ok:
        assert r.returncode == 0, (r.returncode, r.stdout[-3000:], r.stderr[-3000:])
    return r


def read_cor(path: Path, fft: int):
    b = path.read_bytes()
    assert b[:4] == bytes([0x83, 0xF9, 0xA2, 0x3E])
    nsec = int.from_bytes(b[28:32], "little", signed=True)
    rec = 128 + fft // 2 * 8
    assert len(b) == 256 + nsec * rec
    return [np.frombuffer(b[256 + k * rec + 128:256 + (k + 1) * rec], np.float32)
            .reshape(-1, 2).astype(np.float64) @ np.array([1.0, 1j]) for k in range(nsec)]


def library_sectors(engine, scan, raw1, raw2, starts, counts):
    """The library on the derived configuration and the bytes the tool reads
    (from the word-aligned starts), one fxc_sector_submit/wait per sector."""
    b1, b2 = scan.bpf(scan.bits1), scan.bpf(scan.bits2)
    s = engine.open_scan(to_fxc(scan))
    out, first = [], 0
    for nf in counts:
        r1 = raw1[starts[0] + first * b1: starts[0] + (first + nf) * b1]
        r2 = raw2[starts[1] + first * b2: starts[1] + (first + nf) * b2]
        assert r1.size == nf * b1 and r2.size == nf * b2
        out.append((s.wait(s.submit(r1, r2, nf, first)), first, nf, r1, r2))
        first += nf
    s.close()
    return out


def inv_norm(levels, nf, fft):
    p = float(np.mean(np.square(levels)))
    return 1.0 / (0.5 * p * nf * float(fft) ** 2)  # main.rs:2645-2683


def check_cor_files(cor_dir, names, fft, lib, levels, scan, fp64_sectors=()):
    """The .cor spectra equal the library's normalised accumulators (bit for
    bit) and, for the sectors listed, are within tolerance of FP64."""
    spec = {k: read_cor(cor_dir / n, fft) for k, n in names.items()}
    for k in spec:
        assert len(spec[k]) == len(lib), k
    for si, (res, first, nf, r1, r2) in enumerate(lib):
        inv = inv_norm(levels, nf, fft)
        for key in ("acf11", "acf22", "xcf"):
            want = (res[key][: fft // 2] * inv).astype(np.complex64)
            assert np.array_equal(spec[key][si].astype(np.complex64), want), (si, key)
        if si in fp64_sectors:
            ref = oracle.fp64_sector_corr_parallel(scan, r1, r2, nf, first_frame=first)
            for key in ("acf11", "acf22"):
                rel = spectral_errors(spec[key][si], ref[key][: fft // 2] * inv)[0]
                assert rel < 1e-5, (si, key, rel)
            rel, ph, _ = spectral_errors(spec["xcf"][si], ref["xcf"][: fft // 2] * inv,
                                         xcf_floor(ref, nf)[: fft // 2] * inv)
            assert rel < 1e-5 and ph < 1e-4, (si, rel, ph)
    return spec


def test_fft1024_geometry_end_to_end(tmp_path, engine, tool):
    fs, fft, obs_hz, lag = 32e6, 1024, 8.4e9, 123.4
    st1 = Station("YAMAGU32", "A", POS1)
    st2 = Station("YAMAGU34", "B", offset(POS1, (-40.0, -60.0, 70.0)), 1.5e-6, 1e-12)
    assert abs(math.dist(st1.pos, st2.pos) - 100.0) < 5.0
    ra, dec = "12h00m00.0s", "+30d00m00.0s"
    n = int(1.1 * fs) // fft * fft
    nbytes = n * 2 // 8
    kw = dict(st1=st1, st2=st2, fs=fs, obs_hz=obs_hz, fft=fft, bits=2, levels=LEVELS2,
              ext_shuffle=IDENT_EXT, lsb1=False, lsb2=False, epoch=EPOCH, ra=ra, dec=dec,
              length_s=1.0, f1_len=nbytes, f2_len=nbytes,
              products=oracle.PROD_ACF | oracle.PROD_XCF)
    scan, starts, counts, ex = derive(tool, **kw)
    assert abs(ex["gd0"]) > 1e-8, ex  # the baseline delay is live (up to 334 ns)
    # station 2 receives the common component LAG samples after the clock
    # and geometric delays the correlator removes
    x1, x2 = oracle.synth_station_pair(n, 2024, rho=0.05,
                                       delay_samples=lag + (1.5e-6 + ex["gd0"]) * fs)
    ident = list(range(32))
    raw1 = oracle.encode_station(x1, 2, LEVELS2, ident, False)
    raw2 = oracle.encode_station(x2, 2, LEVELS2, ident, False)
    rd = tmp_path / "raw"
    rd.mkdir()
    (rd / f"YAMAGU32_{TAG}.raw").write_bytes(raw1.tobytes())
    (rd / f"YAMAGU34_{TAG}.raw").write_bytes(raw2.tobytes())
    sched = tmp_path / "sched.xml"
    sched.write_text(schedule_xml(st1, st2, fs, 2, LEVELS2, IDENT_EXT, obs_hz, fft, EPOCH, 1.0,
                                  ra, dec))
    out = tmp_path / "cor"
    r = run_tool("yi-corr", "--sc", sched, "--raw", rd, "--cor", out, "--sideband", "USB")
    assert "1-second geometric-delay table enabled" in r.stdout
    names = {"acf11": f"YAMAGU32_YAMAGU32_{TAG}_cli.cor", "xcf": f"YAMAGU32_YAMAGU34_{TAG}_cli.cor",
             "acf22": f"YAMAGU34_YAMAGU34_{TAG}_cli.cor"}
    lib = library_sectors(engine, scan, raw1, raw2, starts, counts)
    spec = check_cor_files(out, names, fft, lib, LEVELS2, scan, fp64_sectors=(0,))
    k = np.arange(20, 490)
    phase = np.unwrap(np.angle(spec["xcf"][0][k]))
    got_lag = abs(np.polyfit(k, phase, 1)[0]) * fft / (2 * np.pi)
    assert abs(got_lag - lag) < 0.5, got_lag


def test_full_rate_configuration_end_to_end(tmp_path, engine, tool):
    fs, fft, obs_hz = 1024e6, 8192, 8.4e9
    ext = oracle.random_shuffle(2468)
    st1 = Station("YAMAGU32", "A", POS1, 0.0, 0.0, rotation_hz=0.0)
    st2 = Station("YAMAGU34", "B", offset(POS1, (155.0, -210.0, 75.0)), 2.5e-7, 3e-13,
                  rotation_hz=16e6)
    ra, dec = "03h30m00.0s", "+20d00m00.0s"
    length = 1.5
    n = int((length + 0.02) * fs) // 16 * 16
    nbytes = n * 2 // 8
    kw = dict(st1=st1, st2=st2, fs=fs, obs_hz=obs_hz, fft=fft, bits=2, levels=LEVELS2,
              ext_shuffle=ext, lsb1=True, lsb2=False, epoch=EPOCH, ra=ra, dec=dec,
              length_s=length, f1_len=nbytes, f2_len=nbytes,
              products=oracle.PROD_ACF | oracle.PROD_XCF, resdelay=0.3, resrate=0.01)
    scan, starts, counts, ex = derive(tool, **kw)
    assert len(counts) == 2 and abs(scan.band[0]) == 128, (counts, scan.band)
    assert abs(ex["geometric_rate_hz"]) > 0.05, ex  # a live geometric fringe rate
    raw1, raw2 = oracle.synth_packed_pair(n, 99, 2, LEVELS2, scan.shuffle1, True, scan.shuffle2,
                                          False, rho=0.05, lag=3)
    rd = tmp_path / "raw"
    rd.mkdir()
    raw1.tofile(rd / f"YAMAGU32_{TAG}.raw")
    raw2.tofile(rd / f"YAMAGU34_{TAG}.raw")
    sched = tmp_path / "sched.xml"
    sched.write_text(schedule_xml(st1, st2, fs, 2, LEVELS2, ext, obs_hz, fft, EPOCH, length, ra,
                                  dec))
    out = tmp_path / "cor"
    run_tool("yi-corr", "--sc", sched, "--raw", rd, "--cor", out, "--sideband",
             "ant1:LSB ant2:USB", "--resdelay", "0.3", "--resrate", "0.01")
    names = {"acf11": f"YAMAGU32_YAMAGU32_{TAG}_cli.cor", "xcf": f"YAMAGU32_YAMAGU34_{TAG}_cli.cor",
             "acf22": f"YAMAGU34_YAMAGU34_{TAG}_cli.cor"}
    lib = library_sectors(engine, scan, raw1, raw2, starts, counts)
    check_cor_files(out, names, fft, lib, LEVELS2, scan, fp64_sectors=(1,))
    print(f"full-rate drop-in: total fringe rate {ex['total_rate_hz']:.4f} Hz "
          f"(geometric {ex['geometric_rate_hz']:.4f} Hz), sectors {counts}, band {scan.band}")


def test_unaligned_start_and_truncated_file(tmp_path, engine, tool):
    fs, fft, obs_hz = 32e6, 1024, 8.4e9
    st1 = Station("YAMAGU32", "A", POS1)
    ra, dec = "12h00m00.0s", "+30d00m00.0s"
    n1 = int(1.1 * fs) // fft * fft
    n2 = int(0.73 * fs)  # station 2 ends mid-frame and mid-word
    b1, b2 = n1 * 2 // 8, n2 * 2 // 8 + 3
    base = dict(fs=fs, obs_hz=obs_hz, fft=fft, bits=2, levels=LEVELS2, ext_shuffle=IDENT_EXT,
                lsb1=False, lsb2=False, epoch=EPOCH, ra=ra, dec=dec, length_s=1.0, f1_len=b1,
                f2_len=b2, products=oracle.PROD_ACF | oracle.PROD_XCF)
    # choose the clock offset so that station 2's desired start is 9 samples
    # into a 16-sample word
    probe = Station("YAMAGU34", "B", offset(POS1, (-40.0, -60.0, 70.0)), 1.5e-6)
    ex0 = derive(tool, st1=st1, st2=probe, **base)[3]
    want = (ex0["start2"] // 16) * 16 + 9
    clock2 = 1.5e-6 + (want - ex0["net_d0"] * fs) / fs
    st2 = Station("YAMAGU34", "B", probe.pos, clock2)
    scan, starts, counts, ex = derive(tool, st1=st1, st2=st2, **base)
    assert ex["start2"] % 16 == 9 and ex["start2_aligned"] == ex["start2"] - 9, ex
    # whole frames of the shorter stream: station 2's samples after its start
    assert ex["total_f"] == (b2 * 8 // 2 - ex["start2"]) // fft, ex
    x1, x2 = oracle.synth_station_pair(n1, 77, rho=0.1, delay_samples=5.2 + clock2 * fs)
    raw1 = oracle.encode_station(x1, 2, LEVELS2, list(range(32)), False)
    raw2 = oracle.encode_station(x2, 2, LEVELS2, list(range(32)), False)[:b2]
    rd = tmp_path / "raw"
    rd.mkdir()
    (rd / f"YAMAGU32_{TAG}.raw").write_bytes(raw1.tobytes())
    (rd / f"YAMAGU34_{TAG}.raw").write_bytes(raw2.tobytes())
    sched = tmp_path / "sched.xml"
    sched.write_text(schedule_xml(st1, st2, fs, 2, LEVELS2, IDENT_EXT, obs_hz, fft, EPOCH, 1.0,
                                  ra, dec))
    out = tmp_path / "cor"
    r = run_tool("yi-corr", "--sc", sched, "--raw", rd, "--cor", out, "--sideband", "USB")
    assert "Word-aligned seek residual: ant1=0 sample(s), ant2=-9 sample(s)" in r.stdout
    names = {"acf11": f"YAMAGU32_YAMAGU32_{TAG}_cli.cor", "xcf": f"YAMAGU32_YAMAGU34_{TAG}_cli.cor",
             "acf22": f"YAMAGU34_YAMAGU34_{TAG}_cli.cor"}
    lib = library_sectors(engine, scan, raw1, raw2, starts, counts)
    check_cor_files(out, names, fft, lib, LEVELS2, scan, fp64_sectors=(0,))


def test_reader_error_aborts_the_run(tmp_path, engine):
    fs, fft = 32e6, 1024
    st1 = Station("YAMAGU32", "A", POS1)
    st2 = Station("YAMAGU34", "B", offset(POS1, (-40.0, -60.0, 70.0)))
    rd = tmp_path / "raw"
    rd.mkdir()
    (rd / f"YAMAGU32_{TAG}.raw").mkdir()  # opens, but every read fails (EISDIR)
    x1, x2 = oracle.synth_station_pair(int(0.2 * fs), 5)
    (rd / f"YAMAGU34_{TAG}.raw").write_bytes(
        oracle.encode_station(x2, 2, LEVELS2, list(range(32)), False).tobytes())
    sched = tmp_path / "sched.xml"
    sched.write_text(schedule_xml(st1, st2, fs, 2, LEVELS2, IDENT_EXT, 8.4e9, fft, EPOCH, 1.0,
                                  "12h00m00.0s", "+30d00m00.0s"))
    r = run_tool("yi-corr", "--sc", sched, "--raw", rd, "--cor", tmp_path / "cor", "--sideband",
                 "USB", ok=False)
    assert r.returncode == 1, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    err = r.stderr.strip().splitlines()[-1]
    assert err.startswith('Error: Custom { kind: Other, error: "synth reader error: '), err
    assert ("failed reading ant1 input: Is a directory (os error 21)" in err
            or "failed to open/seek" in err), err
