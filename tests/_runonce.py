"""The scan configuration run_once derives from a schedule and the command
line (src/main.rs:1063-1212, 1270-1328, 1570-1673, 2058-2072), restated in
Python for the end-to-end tests of the yi-* tools: the test derives the
scan independently of the tool, hands it to the library, and expects the
tool's .cor spectra to be the library's numbers bit for bit.

Only the geometry (precession, sidereal time, baseline delay) comes from the
tools' own geometry code, through tests/cli_host_check.cpp: it is checked on
its own against the reference's geometry tests and published examples
(tests/test_cli_host.py).  Every other value follows the reference's
arithmetic in the reference's operation order, so that the f64 results are
identical."""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

import oracle


def rust_round(x: float) -> float:
    """f64::round: half away from zero."""
    r = math.floor(abs(x))
    if abs(x) - r >= 0.5:
        r += 1.0
    return math.copysign(r, x)


@dataclass
class Station:
    name: str
    key: str
    pos: tuple
    clock_delay: float = 0.0
    clock_rate: float = 0.0
    rotation_hz: float | None = None


def schedule_xml(st1: Station, st2: Station, fs: float, bits: int, levels, ext_shuffle,
                 obs_hz: float, fft: int, epoch: str, length_s: float, ra: str, dec: str,
                 label: str = "cli", skip_s: float | None = None) -> str:
    """A schedule in the reference's XML format (src/xml.rs:66-348, template
    at src/xml.rs:392-420): stations, clocks, terminals, the shuffle (ant1's
    is used for both, a quirk of run_once), source, stream with per-station
    <special> rotations, one process."""
    lv = ",".join(f"{v:+g}" for v in levels)
    sh = ",".join(str(v) for v in ext_shuffle)

    def station(s, term):
        x, y, z = s.pos
        return (f'  <station key="{s.key}"><name>{s.name}</name><pos-x>{x!r}</pos-x>'
                f"<pos-y>{y!r}</pos-y><pos-z>{z!r}</pos-z><terminal>{term}</terminal></station>\n")

    def special(s):
        if s.rotation_hz is None:
            return ""
        return f'    <special key="{s.key}"><rotation>{s.rotation_hz!r}</rotation></special>\n'

    skip = "" if skip_s is None else f"<skip>{skip_s!r}</skip>"
    return (
        '<?xml version="1.0"?>\n<schedule>\n'
        + station(st1, "t1") + station(st2, "t2")
        + f'  <clock key="{st1.key}"><delay>{st1.clock_delay!r}</delay><rate>{st1.clock_rate!r}'
          f"</rate></clock>\n"
        + f'  <clock key="{st2.key}"><delay>{st2.clock_delay!r}</delay><rate>{st2.clock_rate!r}'
          f"</rate></clock>\n"
        + f'  <terminal name="t1"><speed>{int(fs)}</speed><bit>{bits}</bit><level>{lv}</level>'
          "</terminal>\n"
        + f'  <terminal name="t2"><speed>{int(fs)}</speed><bit>{bits}</bit><level>{lv}</level>'
          "</terminal>\n"
        + f'  <shuffle key="{st1.key}">{sh}</shuffle>\n  <shuffle key="{st2.key}">{sh}</shuffle>\n'
        + f'  <source name="SRC"><ra>{ra}</ra><dec>{dec}</dec></source>\n'
        + f"  <stream><label>{label}</label><frequency>{int(obs_hz)}</frequency><fft>{fft}</fft>\n"
        + special(st1) + special(st2)
        + "  </stream>\n"
        + f"  <process><epoch>{epoch}</epoch>{skip}<length>{length_s!r}</length><object>SRC</object>"
          f"<stations>{st1.key}{st2.key}</stations></process>\n"
        + "</schedule>\n")


def derive(tool, *, st1: Station, st2: Station, fs: float, obs_hz: float, fft: int, bits: int,
           levels, ext_shuffle, lsb1: bool, lsb2: bool, epoch: str, ra: str, dec: str,
           length_s: float, f1_len: int, f2_len: int, products: int, skip_s: float = 0.0,
           resdelay: float = 0.0, resrate: float = 0.0, delay: float = 0.0, rate: float = 0.0):
    """Returns (oracle.Scan, start byte of each station, sector frame counts,
    extras) for a one-process schedule run without --length/--skip."""
    obs_mhz = abs(obs_hz) / 1e6                                   # xml.rs:164
    internal = oracle.parse_shuffle(ext_shuffle)                  # args.rs:202-210
    # geometry (main.rs:1101-1118): J2000 input precessed to the epoch
    ra_raw, dec_raw = float(tool("ra", ra)), float(tool("dec", dec))
    mjd = float(tool("mjd", epoch))
    ra_p, dec_p = map(float, tool("precess", repr(ra_raw), repr(dec_raw), repr(mjd)).split())

    def geodelay(m):
        return list(map(float, tool("geodelay", *map(repr, st1.pos), *map(repr, st2.pos),
                                    repr(ra_p), repr(dec_p), repr(m)).split()))

    _, _, gd0, gr0, ga0 = geodelay(mjd)
    # clocks (main.rs:1119-1172, no <clock><epoch>)
    c1d, c1r, c2d, c2r = st1.clock_delay, st1.clock_rate, st2.clock_delay, st2.clock_rate
    clock_delay_s = c2d - c1d
    clock_rate_sps = c2r - c1r
    coarse = 0.0                                                  # main.rs:32
    delay_user = delay + resdelay
    rate_user = rate + resrate
    net_d_rel_no_clock0 = gd0 + coarse + delay_user / fs
    net_d0 = net_d_rel_no_clock0 + clock_delay_s
    # rotations and band alignment (main.rs:1183-1212)
    rot1 = st1.rotation_hz or 0.0
    rot2 = st2.rotation_hz or 0.0
    bw = fs / 2e6
    a1_low, a2_low = obs_mhz + rot1 / 1e6, obs_mhz + rot2 / 1e6
    lo1, lo2 = a1_low * 1e6, a2_low * 1e6
    band = oracle.c_band_alignment(fft, fs, a1_low + 0.5 * bw, a2_low + 0.5 * bw, bw, bw)
    grid = 0 if abs(rot1) <= abs(rot2) else 1
    # scan window (main.rs:1276-1304)
    total_skip = skip_s
    ts1, ts2 = f1_len * 8 // bits, f2_len * 8 // bits
    init = int(rust_round(net_d0 * fs))
    seek1, seek2 = (-init if init < 0 else 0), (init if init > 0 else 0)
    skip_samples = int(rust_round(total_skip * fs))
    start1, start2 = seek1 + skip_samples, seek2 + skip_samples
    avail = min(max(ts1 - start1, 0), max(ts2 - start2, 0))
    available_sec = avail / fs
    requested = max(length_s - total_skip, 0.0)
    total_sec = min(requested, available_sec)
    total_f = int(math.floor(total_sec * fs / fft))
    # rates (main.rs:1316-1328)
    geometric_rate_hz = -1.0 * gr0 * obs_mhz * 1e6
    clock_rate_hz = clock_rate_sps * obs_mhz * 1e6
    df = fs / fft
    rotation_residual = (rot1 - rot2) - band[0] * df
    rotation_fringe = -rotation_residual
    total_rate_hz = geometric_rate_hz + clock_rate_hz + rotation_fringe + rate_user
    # word-aligned starts (main.rs:1577-1616)
    spw = 32 // bits
    s1a, s2a = start1 // spw * spw, start2 // spw * spw
    d_seek = float(s2a - s1a) / fs
    # delay model (main.rs:1618-1673)
    frame_dt = fft / fs
    net_d1_base = net_d_rel_no_clock0 + clock_delay_s - d_seek
    rate_rel = (geometric_rate_hz + rotation_fringe + rate_user) / (obs_mhz * 1e6)
    total_rate1_base = rate_rel + clock_rate_sps
    total_accel1_base = -1.0 * ga0
    n_update = int(max(math.ceil(total_f * frame_dt), 1.0))
    table = np.array([geodelay(mjd + (total_skip + float(sec)) / 86400.0)[2]
                      for sec in range(n_update + 1)])
    extra_rate = (rotation_fringe + rate_user) / (obs_mhz * 1e6)
    dly = dict(frame_dt=frame_dt, fs=fs, time_offset_s=total_skip, coarse_delay_s=coarse,
               delay_user_samples=delay_user, extra_delay_rate_sps=extra_rate,
               clock1_delay_s=c1d, clock1_rate_sps=c1r, clock2_delay_s=c2d, clock2_rate_sps=c2r,
               d_seek=d_seek, net_d1_base=net_d1_base, total_rate1_base=total_rate1_base,
               total_accel1_base=total_accel1_base, net_d2_base=0.0, total_rate2_base=0.0,
               total_accel2_base=0.0, lo1_hz=lo1, lo2_hz=lo2)
    scan = oracle.Scan(fft=fft, fs=fs, bits1=bits, bits2=bits, levels1=list(levels),
                       levels2=list(levels), shuffle1=internal, shuffle2=internal, lsb1=lsb1,
                       lsb2=lsb2, band=tuple(band), grid=grid, products=products, delay=dly,
                       geom_table=table)
    # sector plan (main.rs:2058-2072)
    sectors = int(max(rust_round(total_f * frame_dt), 1.0))
    sectors = min(sectors, max(total_f, 1))
    counts = [total_f // sectors + (1 if si < total_f % sectors else 0) for si in range(sectors)]
    counts = [c for c in counts if c]
    extras = dict(gd0=gd0, gr0=gr0, total_rate_hz=total_rate_hz,
                  geometric_rate_hz=geometric_rate_hz, start1=start1, start2=start2,
                  start1_aligned=s1a, start2_aligned=s2a, total_f=total_f, net_d0=net_d0)
    return scan, (s1a * bits // 8, s2a * bits // 8), counts, extras
