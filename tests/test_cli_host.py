"""Host logic of the yi-* tools on the CPU: the reference's own geometry
tests (src/geom.rs:387-437), published epoch / sidereal-time / precession
examples, .cor header layout (src/cor.rs:152-296), command-line rules
(src/args.rs) and the XML schedule reader (src/xml.rs:66-348)."""
from __future__ import annotations

import math
import shutil
import struct
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "fx-corr_b200" / "cli"


# ------------------------------------------------------------ src/geom.rs tests

def test_reference_geom_tests(tool):
    assert abs(float(tool("ra", "16h42m58.8s")) - float(tool("ra", "164258.8"))) < 1e-12
    assert abs(float(tool("dec", "+39d48m36.0s")) - float(tool("dec", "+394836.0"))) < 1e-12
    assert abs(float(tool("mjd", "2000")) - 51544.5) < 1e-9
    assert abs(float(tool("mjd", "60350.25")) - 60350.25) < 1e-12
    assert abs(float(tool("mjd", "2025-09-29T08:38:00Z")) - 60947.35972222222) < 1e-9
    assert abs(float(tool("mjd", "2024/043 15:52:00")) - 60352.66111111111) < 1e-9
    g0 = float(tool("gmst", 60352.66111))
    g1 = float(tool("gmst", 60352.66111 + 1.0 / 86400.0))
    d = (g1 - g0) % (2 * math.pi)
    assert 7.2e-5 < d < 7.4e-5


def test_coordinate_forms(tool):
    ra = float(tool("ra", "16h42m58.8s"))
    assert abs(ra - math.radians((16 + 42 / 60 + 58.8 / 3600) * 15)) < 1e-12
    assert abs(float(tool("ra", "16:42:58.8")) - ra) < 1e-12
    dec = float(tool("dec", "-39d48m36.0s"))
    assert abs(dec + math.radians(39 + 48 / 60 + 36 / 3600)) < 1e-12
    assert tool("ra", "nonsense").startswith("ERROR")


def test_published_sidereal_time(tool):
    # Meeus, Astronomical Algorithms, example 12.a: 1987 April 10, 0h UT
    # (MJD 46895.0): mean 13h10m46.3668s, apparent 13h10m46.1351s.
    mean = float(tool("gmst", 46895.0))
    app = float(tool("gast", 46895.0))
    hms = lambda h, m, s: (h + m / 60 + s / 3600) * 15 * math.pi / 180
    assert abs(mean - hms(13, 10, 46.3668)) < 2e-5
    assert abs(app - hms(13, 10, 46.1351)) < 4e-6


def test_published_precession(tool):
    # Meeus example 21.b: theta Persei J2000 (41.054063, +49.227750 deg) to
    # 2028 Nov 13.19 TD (JD 2462088.69): (41.547214, +49.348483 deg).
    ra, dec = map(float, tool("precess", math.radians(41.054063), math.radians(49.227750),
                              62088.19).split())
    assert abs(math.degrees(ra) - 41.547214) < 3e-6
    assert abs(math.degrees(dec) - 49.348483) < 3e-6


def test_baseline_delay_properties(tool):
    a = (-3502544.587, 3950966.235, 3566381.192)
    b = (-3502567.576, 3950885.734, 3566449.115)
    blen = math.dist(a, b)
    out = list(map(float, tool("geodelay", *a, *b, 1.2, 0.5, 60352.66).split()))
    rev = list(map(float, tool("geodelay", *b, *a, 1.2, 0.5, 60352.66).split()))
    d, rate, acc = out[2], out[3], out[4]
    assert abs(d) <= blen / 299792458.0
    assert abs(rate) <= 7.3e-5 * blen / 299792458.0 * 1.01
    assert abs(d + rev[2]) < 1e-18 and abs(rate + rev[3]) < 1e-20
    zero = list(map(float, tool("geodelay", *a, *a, 1.2, 0.5, 60352.66).split()))
    assert zero[2] == 0.0 and zero[3] == 0.0


def test_epoch_tags(tool):
    u = int(tool("unix", "2024/043 15:52:00"))
    assert u == 1707753120
    assert tool("tag", u) == "2024043155200"
    assert tool("tag", 0) == "1970001000000"


# ------------------------------------------------------------ .cor headers

def test_cor_file_header_layout(tool):
    h = bytes.fromhex(tool("header"))
    assert len(h) == 256
    assert h[:4] == bytes([0x83, 0xF9, 0xA2, 0x3E])
    ver, one, fs = struct.unpack_from("<iii", h, 4)
    assert (ver, one, fs) == (0x01030000, 1, 1024000000)
    assert struct.unpack_from("<d", h, 16)[0] == 8.4e9
    assert struct.unpack_from("<ii", h, 24) == (8192, 10)
    assert h[32:48].rstrip(b"\0") == b"YAMAGU32" and h[72:73] == b"A"
    assert struct.unpack_from("<ddd", h, 48) == (-3502544.587, 3950966.235, 3566381.192)
    assert h[80:96].rstrip(b"\0") == b"YAMAGU34" and h[120:121] == b"B"
    assert h[128:144].rstrip(b"\0") == b"3C273"
    assert struct.unpack_from("<dd", h, 144) == (3.25, 0.035)
    assert struct.unpack_from("<II", h, 160) == (1707753120, 0)
    assert struct.unpack_from("<II", h, 208) == (1707753120, 0)
    assert h[168:208] == bytes(40) and h[216:256] == bytes(40)


@pytest.mark.parametrize("ts,integ", [(1707753120, 1.0), (1707753121, 0.999424), (5, -1.0)])
def test_cor_sector_header(tool, ts, integ):
    h = bytes.fromhex(tool("sector", ts, integ))
    assert len(h) == 128
    f32 = struct.unpack("<f", struct.pack("<f", integ))[0]
    it = f32 if (math.isfinite(f32) and f32 > 0) else 1.0
    end = ts + it
    nsec = (end - math.trunc(end)) * 1e9
    sec = math.floor(end)
    st, st_ns, et, et_ns = struct.unpack_from("<iIII", h, 0)
    assert (st, st_ns) == (ts, 0)
    assert (et, et_ns) == (sec, round(nsec))
    assert struct.unpack_from("<f", h, 112)[0] == f32
    assert h[16:112] == bytes(96) and h[116:] == bytes(12)


# ------------------------------------------------------------ command line

def parse(tool, *argv):
    out = tool("args", *argv)
    if out.startswith("ARGSEXIT"):
        return out
    return dict(line.split("=", 1) for line in out.splitlines() if "=" in line and " " not in
                line.split("=", 1)[0])


def test_args_aliases_prefixes_and_values(tool):
    a = parse(tool, "--sc", "s.xml", "--data", "d", "--output", "o", "--bit", "ant1:2", "ant2:4",
              "--level", "-1.5", "-0.5", "0.5", "1.5", "--dec", "-30d00m00s", "--rotation",
              "ant1:-5e6", "ant2:0", "--delay", "-3.5", "--coarse=-1e-6", "--fft", "8192")
    assert a["schedule"] == "s.xml" and a["raw"] == "d" and a["cor"] == "o"
    assert a["bin"] == "ant1:2;ant2:4"
    assert a["level"] == "-1.5;-0.5;0.5;1.5"
    assert a["dec"] == "-30d00m00s"
    assert a["rotation"] == "ant1:-5e6;ant2:0"
    assert float(a["delay"]) == -3.5 and float(a["coarse"]) == -1e-6
    assert a["fft"] == "8192"
    assert a["sideband"] == "LSB"  # default_value
    b = parse(tool, "--schedule", "x.xml", "--raw-dir", "r", "--cor-dir", "c", "--samp", "512",
              "--sideband", "ant1:LSB", "ant2:USB")
    assert b["raw"] == "r" and b["cor"] == "c" and float(b["sampling"]) == 512.0
    assert b["sideband"] == "ant1:LSB;ant2:USB"


@pytest.mark.parametrize("argv,code,msg", [
    ((), 2, "Usage"),
    (("--r", "x"), 2, "matches more than one"),
    (("--fft", "abc"), 2, "invalid value 'abc'"),
    (("--fft", "1024", "--fft", "2048"), 2, "cannot be used multiple times"),
    (("--ra",), 2, "a value is required"),
    (("--obsfreq", "-5"), 2, "a value is required"),
    (("--bogus",), 2, "unexpected argument '--bogus'"),
    (("stray",), 2, "unexpected argument 'stray'"),
    (("--mkxml=1",), 2, "unexpected value"),
    (("--help",), 0, "yi-corr: auto + cross correlation"),
    (("--delay-reference", "ant3"), 2, "possible values"),
])
def test_args_errors(tool, argv, code, msg):
    out = parse(tool, *argv)
    assert isinstance(out, str) and out.startswith(f"ARGSEXIT {code}"), out
    assert msg in out, out


def test_levels_shuffle_per_antenna(tool):
    assert tool("levels", 2, "-3,-1,1,3") == "-3 -1 1 3"
    assert tool("levels", 2, "-3,-1,1").startswith("ERROR Expected 4 levels, received 3")
    assert tool("levels", 1, "-1,x").startswith("ERROR")
    ext = ",".join(str(31 - i) for i in range(32))
    assert tool("shuffle", ext) == " ".join(str(i) for i in range(32))
    swap = ",".join(str(v) for v in [30, 31, 28, 29] + list(range(27, -1, -1)))
    internal = list(map(int, tool("shuffle", swap).split()))
    assert internal[31] == 30 and internal[30] == 31 and internal[27] == 27
    assert tool("shuffle", "0,1,2").startswith("ERROR Shuffle map must contain exactly 32")
    assert tool("shuffle", ",".join(["0"] * 32)).startswith("ERROR Shuffle map must be a permutation")
    assert tool("perant", "D", "ant1:A ant2:B") == "A|B"
    assert tool("perant", "D", "ant2:B") == "D|B"
    assert tool("perant", "D", "X") == "X|X"
    assert tool("perant", "D", "ant1:A,Y") == "Y|Y"  # bare values in a tagged entry set both
    assert tool("perant", "D") == "D|D"


def test_phased_weights(tool):
    assert float(tool("weight", 100, 2, 0, 0, 0.65)) == 2 / 100
    assert abs(float(tool("weight", 100, 1, 2000, 0, 0.65)) - 1 / 2000) < 1e-18
    kb, jy = 1.380649e-23, 1e26
    area = 0.65 * math.pi * (32 / 2) ** 2
    sefd = 2 * kb * 50 / area * jy
    assert abs(float(tool("weight", 50, 1, 0, 32, 0.65)) - 1 / sefd) < 1e-15
    assert tool("weight", 0, 1, 0, 0, 0.65).startswith("ERROR A1 Tsys must be non-zero")


# ------------------------------------------------------------ XML schedule

def test_example_xml_round_trip(tool, tmp_path):
    p = tmp_path / "example.xml"
    tool("mkxml", p)
    out = tool("xml", p)
    assert "names=ANT1,ANT2 keys=A,B" in out
    assert "fs=1024000000 obs_mhz=8400 fft=16384" in out
    assert "bits=2,2 level=-1.5,-0.5,+0.5,+1.5" in out
    assert "processes=1" in out


def test_xml_schedule_fields(tool, tmp_path):
    ident = ",".join(str(31 - i) for i in range(32))
    xml = f"""<?xml version="1.0"?>
<!-- comment -->
<schedule>
  <station key="X"><name>FAR</name><terminal>tx</terminal></station>
  <station key="A"><name>STA</name><pos-x>1</pos-x><pos-y>2</pos-y><pos-z>3</pos-z><terminal>ta</terminal></station>
  <station key="B"><name>STB</name><terminal>tb</terminal></station>
  <clock key="A"><delay>1e-6</delay><rate>0</rate></clock>
  <clock key="B"><delay>3e-6</delay><rate>2e-12</rate><epoch>2024/043 00:00:00</epoch></clock>
  <terminal name="ta"><speed>512000000</speed><bit>2</bit><level>-3,-1,1,3</level></terminal>
  <terminal name="tb"><speed>256000000</speed><bit>4</bit></terminal>
  <shuffle key="A">{ident}</shuffle>
  <source name="S1"><ra>01h00m00s</ra><dec>+10d00m00s</dec></source>
  <source name="S2"><ra>02h00m00s</ra><dec>-20d00m00s</dec></source>
  <stream><label>lab&amp;el</label><frequency>-6.7e9</frequency><fft>4096</fft>
    <special key="A"><rotation>1e6</rotation></special>
    <special key="B"><sideband>usb</sideband><rotation>-2e6</rotation></special></stream>
  <process><epoch>2024/043 15:52:00</epoch><skip>2</skip><length>5</length><object>S2</object><stations>AB</stations></process>
  <process><epoch>2024/043 16:00:00</epoch><object>S1</object><stations>AX</stations></process>
  <process><epoch>2024/043 17:00:00</epoch><object>S1</object><stations>BA</stations></process>
  <process><epoch>2024/043 18:00:00</epoch><fft> 16384 </fft><bit>4</bit><level>-1.5,-0.5,0.5,1.5</level><object>S1</object><stations>AB</stations></process>
</schedule>"""
    p = tmp_path / "s.xml"
    p.write_text(xml)
    out = tool("xml", p)
    assert "ra=02h00m00s dec=-20d00m00s" in out  # the first process's object
    assert "fs=512000000 obs_mhz=6700 fft=4096" in out
    assert "names=STA,STB keys=A,B" in out
    assert "bits=2,4 level=-3,-1,1,3" in out
    assert "sideband=LSB,USB" in out  # negative frequency -> LSB default
    assert "rot=1000000,-2000000" in out
    assert "clock=9.9999999999999995e-07,3.0000000000000001e-06" in out
    # processes without both station keys are dropped (src/xml.rs:265-270)
    assert "processes=3" in out  # the AX process has no station B
    assert "process epoch=2024/043 15:52:00 skip=2 length=5.000000 fft=- bit=- level=-" in out
    # this build's per-process extension (<fft>, <bit>, <level> inside <process>)
    assert ("process epoch=2024/043 18:00:00 skip=0 length=- fft=16384 bit=4 "
            "level=-1.5,-0.5,0.5,1.5") in out
