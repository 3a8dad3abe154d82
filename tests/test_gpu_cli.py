"""The yi-* command line end to end on the GPU: XML schedule + .raw files in,
.cor (and phased .raw) out.  The spectra a tool writes must be the ones the
library computes for the configuration the reference's run_once derives
(bit for bit), and within tolerance of the FP64 oracle after the .cor
normalisation; the XCF phase slope recovers the synthetic lag."""
from __future__ import annotations

import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from _cases import spectral_errors, to_fxc, xcf_floor

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "fx-corr_b200" / "bin"
FS, FFT, OBS_HZ = 32e6, 1024, 8.4e9
CLOCK2_S, CLOCK2_RATE = 1.5e-6, 1e-12
LAG = 123.4
EPOCH, TAG = "2024/043 15:52:00", "2024043155200"
IDENT = ",".join(str(31 - i) for i in range(32))


def write_case(d: Path, seconds=1.1, seed=2024):
    """Schedule (zero-length baseline, so the geometric terms vanish) and two
    .raw files: 2-bit +-1/+-3, common component at rho=0.05 delayed by LAG
    samples plus the 1.5 us clock offset at station 2."""
    xml = f"""<?xml version="1.0"?>
<schedule>
  <station key="A"><name>YAMAGU32</name><pos-x>-3502544.587</pos-x><pos-y>3950966.235</pos-y>
    <pos-z>3566381.192</pos-z><terminal>t1</terminal></station>
  <station key="B"><name>YAMAGU34</name><pos-x>-3502544.587</pos-x><pos-y>3950966.235</pos-y>
    <pos-z>3566381.192</pos-z><terminal>t2</terminal></station>
  <clock key="A"><delay>0</delay><rate>0</rate></clock>
  <clock key="B"><delay>{CLOCK2_S}</delay><rate>{CLOCK2_RATE}</rate></clock>
  <terminal name="t1"><speed>{int(FS)}</speed><bit>2</bit><level>-3,-1,+1,+3</level></terminal>
  <terminal name="t2"><speed>{int(FS)}</speed><bit>2</bit><level>-3,-1,+1,+3</level></terminal>
  <shuffle key="A">{IDENT}</shuffle>
  <shuffle key="B">{IDENT}</shuffle>
  <source name="SRC"><ra>12h00m00.0s</ra><dec>+30d00m00.0s</dec></source>
  <stream><label>cli</label><frequency>{int(OBS_HZ)}</frequency><fft>{FFT}</fft></stream>
  <process><epoch>{EPOCH}</epoch><length>1</length><object>SRC</object>
    <stations>AB</stations></process>
</schedule>
"""
    (d / "sched.xml").write_text(xml)
    raw = d / "raw"
    raw.mkdir()
    n = int(seconds * FS)
    n -= n % FFT
    x1, x2 = oracle.synth_station_pair(n, seed, rho=0.05, delay_samples=LAG + CLOCK2_S * FS)
    lv = oracle.default_levels(2)
    ident = list(range(32))
    (raw / f"YAMAGU32_{TAG}.raw").write_bytes(oracle.encode_station(x1, 2, lv, ident, False).tobytes())
    (raw / f"YAMAGU34_{TAG}.raw").write_bytes(oracle.encode_station(x2, 2, lv, ident, False).tobytes())
    return d / "sched.xml", raw


def run_tool(name, *args, cwd=None):
    r = subprocess.run([str(BIN / name), *map(str, args)], cwd=cwd, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return r


def read_cor(path: Path, fft: int):
    b = path.read_bytes()
    assert b[:4] == bytes([0x83, 0xF9, 0xA2, 0x3E])
    assert int.from_bytes(b[4:8], "little") == 0x01030000
    nsec = int.from_bytes(b[28:32], "little", signed=True)
    rec = 128 + fft // 2 * 8
    assert len(b) == 256 + nsec * rec
    spec = [np.frombuffer(b[256 + k * rec + 128:256 + (k + 1) * rec], np.float32)
            .reshape(-1, 2) for k in range(nsec)]
    return nsec, [s[:, 0] + 1j * s[:, 1] for s in spec]


def derived_scan(total_f, bits_out=2, products=oracle.PROD_ACF | oracle.PROD_XCF):
    """The configuration run_once derives for write_case's schedule
    (src/main.rs:1063-1673): zero geometry, station 2 read 48 samples later,
    clock rate as the only delay rate."""
    seek2 = round(CLOCK2_S * FS)
    d_seek = seek2 / FS
    frame_dt = FFT / FS
    n_table = max(math.ceil(total_f * frame_dt), 1) + 1
    delay = dict(time_offset_s=0.0, clock2_delay_s=CLOCK2_S, clock2_rate_sps=CLOCK2_RATE,
                 d_seek=d_seek, net_d1_base=(0.0 + 0.0 + 0.0 / FS) + CLOCK2_S - d_seek,
                 total_rate1_base=(0.0 + 0.0 + 0.0) / OBS_HZ + CLOCK2_RATE,
                 total_accel1_base=-0.0, lo1_hz=OBS_HZ, lo2_hz=OBS_HZ)
    scan = oracle.Scan(fft=FFT, fs=FS, bits1=2, bits2=2, levels1=oracle.default_levels(2),
                       levels2=oracle.default_levels(2), shuffle1=list(range(32)),
                       shuffle2=list(range(32)), lsb1=False, lsb2=False, band=(0, 0, 512, 0),
                       grid=0, products=products, delay=delay, geom_table=np.zeros(n_table))
    return scan, seek2 * 2 // 8


def test_yi_corr_end_to_end(tmp_path, engine):
    sched, raw = write_case(tmp_path)
    out = tmp_path / "cor"
    run_tool("yi-corr", "--sc", sched, "--raw", raw, "--cor", out, "--sideband", "USB")
    files = {p.name: p for p in out.glob("*.cor")}
    names = [f"YAMAGU32_YAMAGU32_{TAG}_cli.cor", f"YAMAGU32_YAMAGU34_{TAG}_cli.cor",
             f"YAMAGU34_YAMAGU34_{TAG}_cli.cor"]
    assert sorted(files) == sorted(names)
    total_f = int(1.0 * FS / FFT)
    nsec, s11 = read_cor(files[names[0]], FFT)
    _, s12 = read_cor(files[names[1]], FFT)
    _, s22 = read_cor(files[names[2]], FFT)
    assert nsec == 1

    scan, off2 = derived_scan(total_f)
    b = scan.bpf(2)
    r1 = np.fromfile(raw / f"YAMAGU32_{TAG}.raw", np.uint8)[: total_f * b]
    r2 = np.fromfile(raw / f"YAMAGU34_{TAG}.raw", np.uint8)[off2: off2 + total_f * b]
    # the library on the same configuration and bytes: identical numbers
    s = engine.open_scan(to_fxc(scan))
    sid = s.submit(r1, r2, total_f, 0)
    lib = s.wait(sid)
    s.close()
    p = float(np.mean(np.square(oracle.default_levels(2))))
    inv = 1.0 / (0.5 * p * total_f * float(FFT) ** 2)
    for got, ref in ((s11[0], lib["acf11"]), (s22[0], lib["acf22"]), (s12[0], lib["xcf"])):
        want = (ref[: FFT // 2] * inv).astype(np.complex64)
        assert np.array_equal(got.astype(np.complex64), want)
    # and the FP64 oracle within the stated tolerance
    ref = oracle.fp64_sector_corr(scan, r1, r2, total_f, first_frame=0)
    for got, key in ((s11[0], "acf11"), (s22[0], "acf22")):
        rel, ph, ab = spectral_errors(got, ref[key][: FFT // 2] * inv)
        assert rel < 1e-5, (key, rel)
    rel, ph, ab = spectral_errors(s12[0], ref["xcf"][: FFT // 2] * inv,
                                  xcf_floor(ref, total_f)[: FFT // 2] * inv)
    assert rel < 1e-5 and ph < 1e-4, (rel, ph)
    # XCF phase slope across the band: the lag left after the clock correction
    k = np.arange(20, 490)
    phase = np.unwrap(np.angle(s12[0][k]))
    slope = np.polyfit(k, phase, 1)[0]
    lag = abs(slope) * FFT / (2 * np.pi)
    assert abs(lag - LAG) < 0.5, lag


def test_yi_acf_xcf_and_phased(tmp_path, engine):
    sched, raw = write_case(tmp_path, seconds=1.05, seed=7)
    total_f = int(1.0 * FS / FFT)
    out = tmp_path / "cor"
    run_tool("yi-acf", "--sc", sched, "--raw", raw, "--cor", out, "--sideband", "USB")
    acf = sorted(p.name for p in out.glob("*.cor"))
    assert acf == [f"YAMAGU32_YAMAGU32_{TAG}_cli.cor", f"YAMAGU34_YAMAGU34_{TAG}_cli.cor"]
    out2 = tmp_path / "cor2"
    run_tool("yi-xcf", "--sc", sched, "--raw", raw, "--cor", out2, "--sideband", "USB")
    assert sorted(p.name for p in out2.glob("*.cor")) == [f"YAMAGU32_YAMAGU34_{TAG}_cli.cor"]
    # phased: .raw and phased .cor land in the working directory
    work = tmp_path / "work"
    work.mkdir()
    run_tool("yi-phasedarray", "--sc", sched, "--raw", raw, "--sideband", "USB", cwd=work)
    praw = work / f"YAMAGU66_{TAG}.raw"
    pcor = work / f"YAMAGU66_YAMAGU66_{TAG}_phasedarray.cor"
    assert praw.exists() and pcor.exists()
    scan, off2 = derived_scan(total_f, products=oracle.PROD_PHASED | oracle.PROD_RAW)
    b = scan.bpf(2)
    r1 = np.fromfile(raw / f"YAMAGU32_{TAG}.raw", np.uint8)[: total_f * b]
    r2 = np.fromfile(raw / f"YAMAGU34_{TAG}.raw", np.uint8)[off2: off2 + total_f * b]
    s = engine.open_scan(to_fxc(scan))
    sid = s.submit(r1, r2, total_f, 0)
    lib = s.wait(sid)
    s.close()
    assert praw.read_bytes() == lib["raw"].tobytes()
    nsec, sph = read_cor(pcor, FFT)
    p = float(np.mean(np.square(oracle.default_levels(2))))
    inv = 1.0 / (0.5 * max(p + p, 1e-12) * total_f * float(FFT) ** 2)
    assert np.array_equal(sph[0].astype(np.complex64),
                          (lib["phased"][: FFT // 2] * inv).astype(np.complex64))


def test_multi_process_schedule(tmp_path):
    """Two <process> entries run sequentially, one output set each."""
    sched, raw = write_case(tmp_path, seconds=2.2, seed=3)
    x = sched.read_text().replace(
        "</schedule>",
        f"  <process><epoch>{EPOCH}</epoch><skip>1</skip><length>2</length><object>SRC</object>"
        "<stations>AB</stations></process>\n</schedule>")
    sched.write_text(x)
    out = tmp_path / "cor"
    r = run_tool("yi-xcf", "--sc", sched, "--raw", raw, "--cor", out, "--sideband", "USB")
    assert "Processing all scans sequentially: 2 process entries" in r.stdout
    names = sorted(p.name for p in out.glob("*.cor"))
    assert names == [f"YAMAGU32_YAMAGU34_{TAG}_cli.cor", f"YAMAGU32_YAMAGU34_2024043155201_cli.cor"]


def _cor_records(path: Path, fft: int):
    b = path.read_bytes()
    nsec = int.from_bytes(b[28:32], "little", signed=True)
    rec = 128 + fft // 2 * 8
    heads = [b[256 + k * rec:256 + k * rec + 128] for k in range(nsec)]
    return b[:256], heads, read_cor(path, fft)[1]


def test_multi_process_jobs_match_sequential(tmp_path):
    """--jobs (this build's extension) runs the <process> entries at once, their
    sectors computed together by a batched server: the same files with the same
    header bytes, spectra within FP32 rounding of the one-after-another run;
    phased .raw frames (the phased batch kernels) identical byte for byte."""
    sched, raw = write_case(tmp_path, seconds=3.3, seed=5)
    # <length> counts from the epoch, as in the reference: skip k, length k + 1
    procs = "".join(
        f"  <process><epoch>{EPOCH}</epoch><skip>{k}</skip><length>{k + 1}</length>"
        "<object>SRC</object><stations>AB</stations></process>\n" for k in (1, 2))
    sched.write_text(sched.read_text().replace("</schedule>", procs + "</schedule>"))
    seq, par = tmp_path / "seq", tmp_path / "par"
    run_tool("yi-corr", "--sc", sched, "--raw", raw, "--cor", seq, "--sideband", "USB")
    r = run_tool("yi-corr", "--sc", sched, "--raw", raw, "--cor", par, "--sideband", "USB",
                 "--jobs", "3")
    assert "Processing all scans, 3 at a time: 3 process entries" in r.stdout
    names = sorted(p.name for p in seq.glob("*.cor"))
    assert len(names) == 9 and names == sorted(p.name for p in par.glob("*.cor"))
    for name in names:
        h_s, sh_s, sp_s = _cor_records(seq / name, FFT)
        h_p, sh_p, sp_p = _cor_records(par / name, FFT)
        assert h_s == h_p and sh_s == sh_p, name
        for a, b in zip(sp_p, sp_s):
            assert np.max(np.abs(a - b)) <= 1e-5 * np.max(np.abs(b)), name
    # phased outputs go to the working directory
    (tmp_path / "ph_seq").mkdir()
    (tmp_path / "ph_par").mkdir()
    run_tool("yi-phasedarray", "--sc", sched, "--raw", raw, "--sideband", "USB",
             cwd=tmp_path / "ph_seq")
    run_tool("yi-phasedarray", "--sc", sched, "--raw", raw, "--sideband", "USB", "--jobs", "3",
             cwd=tmp_path / "ph_par")
    files = sorted(p.name for p in (tmp_path / "ph_seq").iterdir() if p.is_file())
    assert files and files == sorted(p.name for p in (tmp_path / "ph_par").iterdir()
                                     if p.is_file())
    for name in files:
        a, b = (tmp_path / "ph_seq" / name), (tmp_path / "ph_par" / name)
        if name.endswith(".raw"):  # every frame computed by the same code: identical
            assert a.read_bytes() == b.read_bytes(), name
        else:  # phased power summed per batch item: the same headers, FP32 rounding
            h_s, sh_s, sp_s = _cor_records(a, FFT)
            h_p, sh_p, sp_p = _cor_records(b, FFT)
            assert h_s == h_p and sh_s == sh_p, name
            for x, y in zip(sp_p, sp_s):
                assert np.max(np.abs(x - y)) <= 1e-5 * np.max(np.abs(y)), name


def _derived_mixed(total_f, fft, bits, levels):
    """derived_scan for another FFT length and bit depth (same stations,
    clocks and zero geometry); the reader starts station 2 at the word
    boundary at or before the clock offset (main.rs:1577-1616), the rest of
    the offset stays in the delay model."""
    spw = 32 // bits
    seek2 = round(CLOCK2_S * FS) // spw * spw
    d_seek = seek2 / FS
    n_table = max(math.ceil(total_f * fft / FS), 1) + 1
    delay = dict(time_offset_s=0.0, clock2_delay_s=CLOCK2_S, clock2_rate_sps=CLOCK2_RATE,
                 d_seek=d_seek, net_d1_base=CLOCK2_S - d_seek, total_rate1_base=CLOCK2_RATE,
                 total_accel1_base=-0.0, lo1_hz=OBS_HZ, lo2_hz=OBS_HZ)
    scan = oracle.Scan(fft=fft, fs=FS, bits1=bits, bits2=bits, levels1=list(levels),
                       levels2=list(levels), shuffle1=list(range(32)), shuffle2=list(range(32)),
                       lsb1=False, lsb2=False, band=(0, 0, fft // 2, 0), grid=0,
                       products=oracle.PROD_ACF | oracle.PROD_XCF, delay=delay,
                       geom_table=np.zeros(n_table))
    return scan, seek2 * bits // 8


def test_mixed_fft_and_bits_per_process(tmp_path, engine):
    """Config 4's mixed classes in one schedule, through this build's
    per-process <fft>/<bit>/<level> extension: FFT 1024 / 4096 / 16384 at
    2 / 1 / 4 bits (the last with the default uniform level table).  The
    one-after-another run equals the library on each derived configuration
    bit for bit; the --jobs run (one batched server, three FFT lengths at
    once) matches it within FP32 rounding."""
    sched, raw = write_case(tmp_path, seconds=0.1, seed=9)
    procs = [("2024/043 15:53:00", "2024043155300", 1024, 2, [-3.0, -1.0, 1.0, 3.0], True),
             ("2024/043 15:54:00", "2024043155400", 4096, 1, [-1.0, 1.0], True),
             ("2024/043 15:55:00", "2024043155500", 16384, 4, oracle.default_levels(4), False)]
    xml = sched.read_text()
    a, b = xml.index("<process>"), xml.index("</process>") + len("</process>")
    entries = ""
    for k, (ep, tag, fft, bits, lv, explicit) in enumerate(procs):
        lvs = f"<level>{','.join(f'{x:g}' for x in lv)}</level>" if explicit else ""
        entries += (f"<process><epoch>{ep}</epoch><length>1</length><fft>{fft}</fft>"
                    f"<bit>{bits}</bit>{lvs}<object>SRC</object><stations>AB</stations>"
                    "</process>\n  ")
        n = int(1.1 * FS)
        n -= n % fft
        x1, x2 = oracle.synth_station_pair(n, 40 + k, rho=0.1, delay_samples=LAG + CLOCK2_S * FS)
        ident = list(range(32))
        (raw / f"YAMAGU32_{tag}.raw").write_bytes(
            oracle.encode_station(x1, bits, lv, ident, False).tobytes())
        (raw / f"YAMAGU34_{tag}.raw").write_bytes(
            oracle.encode_station(x2, bits, lv, ident, False).tobytes())
    sched.write_text(xml[:a] + entries + xml[b:])
    seq, par = tmp_path / "seq", tmp_path / "par"
    run_tool("yi-corr", "--sc", sched, "--raw", raw, "--cor", seq, "--sideband", "USB")
    run_tool("yi-corr", "--sc", sched, "--raw", raw, "--cor", par, "--sideband", "USB",
             "--jobs", "3")
    for ep, tag, fft, bits, lv, _ in procs:
        total_f = int(1.0 * FS / fft)
        names = [f"YAMAGU32_YAMAGU32_{tag}_cli.cor", f"YAMAGU32_YAMAGU34_{tag}_cli.cor",
                 f"YAMAGU34_YAMAGU34_{tag}_cli.cor"]
        scan, off2 = _derived_mixed(total_f, fft, bits, lv)
        bpf = scan.bpf(bits)
        r1 = np.fromfile(raw / f"YAMAGU32_{tag}.raw", np.uint8)[: total_f * bpf]
        r2 = np.fromfile(raw / f"YAMAGU34_{tag}.raw", np.uint8)[off2: off2 + total_f * bpf]
        s = engine.open_scan(to_fxc(scan))
        lib = s.wait(s.submit(r1, r2, total_f, 0))
        s.close()
        p = float(np.mean(np.square(lv)))
        inv = 1.0 / (0.5 * p * total_f * float(fft) ** 2)
        for name, key in zip(names, ("acf11", "xcf", "acf22")):
            nsec, got = read_cor(seq / name, fft)
            assert nsec == 1, name
            want = (lib[key][: fft // 2] * inv).astype(np.complex64)
            assert np.array_equal(got[0].astype(np.complex64), want), name
            _, gp = read_cor(par / name, fft)
            assert np.max(np.abs(gp[0] - got[0])) <= 1e-5 * np.max(np.abs(got[0])), name
