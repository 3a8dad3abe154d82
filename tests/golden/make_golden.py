"""Writes tests/golden/kat.json: known-answer vectors for the fx-corr hot path.

The reference ships no fixtures for this path and cannot be built here, so
every expected value below is a literal: derived by hand from the cited
reference lines, or (the `readme` section) a worked example the reference's
README states itself.  Nothing here calls an oracle or the product.
Run:  python tests/golden/make_golden.py
"""
import json
from pathlib import Path

L2 = [-1.5, -0.5, 0.5, 1.5]            # VSREC level order (src/xml.rs:372)
L1 = [-1.0, 1.0]
L4 = [i - 7.5 for i in range(16)]
L8 = [i - 127.5 for i in range(256)]
IDENT = list(range(32))
PAIR = [i ^ 1 for i in range(32)]
# VSREC example (src/xml.rs:376), external MSB-first list
VSREC_EXT = [24, 25, 26, 27, 28, 29, 30, 31, 16, 17, 18, 19, 20, 21, 22, 23,
             8, 9, 10, 11, 12, 13, 14, 15, 0, 1, 2, 3, 4, 5, 6, 7]
# parse_shuffle (args.rs:208): internal[31-idx] = ext[idx] -> bit reversal
# inside every byte: internal[8b + j] = 8b + 7 - j
VSREC_INT = [8 * (o // 8) + 7 - (o % 8) for o in range(32)]
REVERSE = [31 - o for o in range(32)]

decode = [
    # utils.rs:247-299, identity 2-bit LUT path.  LE bytes E4 1B 00 FF:
    # E4 = 11 10 01 00 -> codes 0,1,2,3 ; 1B -> 3,2,1,0 ; 00 -> 0 x4 ; FF -> 3 x4
    dict(name="2bit_identity", bits=2, shuffle=IDENT, levels=L2, lsb=False,
         raw=[0xE4, 0x1B, 0x00, 0xFF], samples=16,
         expect=[-1.5, -0.5, 0.5, 1.5, 1.5, 0.5, -0.5, -1.5,
                 -1.5, -1.5, -1.5, -1.5, 1.5, 1.5, 1.5, 1.5]),
    # same bytes, LSB input: odd samples negated (utils.rs:196-197, 273)
    dict(name="2bit_identity_lsb", bits=2, shuffle=IDENT, levels=L2, lsb=True,
         raw=[0xE4, 0x1B, 0x00, 0xFF], samples=16,
         expect=[-1.5, 0.5, 0.5, -1.5, 1.5, -0.5, -0.5, 1.5,
                 -1.5, 1.5, -1.5, 1.5, 1.5, -1.5, 1.5, -1.5]),
    # utils.rs:162 pair swap: E4 = 11 10 01 00 -> 11 01 10 00 = D8 -> codes 0,2,1,3
    dict(name="2bit_pairswap", bits=2, shuffle=PAIR, levels=L2, lsb=False,
         raw=[0xE4, 0x00, 0x00, 0x00], samples=16,
         expect=[-1.5, 0.5, -0.5, 1.5] + [-1.5] * 12),
    # utils.rs:163-168 generic: VSREC reverses bits in each byte: 01 -> 80 -> codes 0,0,0,2
    dict(name="2bit_vsrec", bits=2, shuffle=VSREC_INT, levels=L2, lsb=False,
         raw=[0x01, 0x00, 0x00, 0x00], samples=16,
         expect=[-1.5, -1.5, -1.5, 0.5] + [-1.5] * 12),
    # utils.rs:231-245 1-bit: word 0x00000005 -> bits 1,0,1,0,...
    dict(name="1bit_identity", bits=1, shuffle=IDENT, levels=L1, lsb=False,
         raw=[0x05, 0x00, 0x00, 0x00], samples=32,
         expect=[1.0, -1.0, 1.0] + [-1.0] * 29),
    # utils.rs:317-332 4-bit: word 0x76543210 -> codes 0..7
    dict(name="4bit_identity", bits=4, shuffle=IDENT, levels=L4, lsb=False,
         raw=[0x10, 0x32, 0x54, 0x76], samples=8,
         expect=[-7.5, -6.5, -5.5, -4.5, -3.5, -2.5, -1.5, -0.5]),
    # utils.rs:333-348 8-bit: bytes 00 01 7F FF -> codes 0,1,127,255
    dict(name="8bit_identity", bits=8, shuffle=IDENT, levels=L8, lsb=False,
         raw=[0x00, 0x01, 0x7F, 0xFF], samples=4,
         expect=[-127.5, -126.5, -0.5, 127.5]),
    # 8-bit with the full reversal shuffle: bit 0 -> bit 31: word 80000000 -> codes 0,0,0,128
    dict(name="8bit_reverse", bits=8, shuffle=REVERSE, levels=L8, lsb=True,
         raw=[0x01, 0x00, 0x00, 0x00], samples=4,
         expect=[-127.5, 127.5, -127.5, -0.5]),
    # identity 2-bit: 3 bytes -> one 2-byte pair (8 samples) + remainder byte (4)
    dict(name="2bit_ragged_remainder", bits=2, shuffle=IDENT, levels=L2, lsb=False,
         raw=[0xE4, 0x00, 0x1B], samples=12,
         expect=[-1.5, -0.5, 0.5, 1.5, -1.5, -1.5, -1.5, -1.5, 1.5, 0.5, -0.5, -1.5]),
    # non-identity 2-bit reads chunks_exact(4): 6 bytes -> 16 samples != 24 -> error
    dict(name="2bit_pairswap_short", bits=2, shuffle=PAIR, levels=L2, lsb=False,
         raw=[0, 0, 0, 0, 0, 0], samples=24, expect=None),
]

shift = [  # utils.rs:126-145
    dict(x=[1, 2, 3, 4], s=1, expect=[0, 1, 2, 3]),
    dict(x=[1, 2, 3, 4], s=-1, expect=[2, 3, 4, 0]),
    dict(x=[1, 2, 3, 4], s=3, expect=[0, 0, 0, 1]),
    dict(x=[1, 2, 3, 4], s=4, expect=[0, 0, 0, 0]),
    dict(x=[1, 2, 3, 4], s=-5, expect=[0, 0, 0, 0]),
    dict(x=[1, 2, 3, 4], s=0, expect=[1, 2, 3, 4]),
]

parse_shuffle = [  # args.rs:202-210
    dict(ext=list(range(31, -1, -1)), expect=IDENT),          # DEFAULT_SHUFFLE_IN
    dict(ext=VSREC_EXT, expect=VSREC_INT),
    dict(ext=[0] * 32, expect=None),                          # not a permutation
]

band = [  # main.rs:363-372 with bw = fs/2e6 and centres c = obs + rot/1e6 + bw/2
    # 1024 Msps, N=8192: df = 125 kHz; 16 MHz offset -> sb = 128; v = min(4097, 4096)
    dict(fft=8192, fs=1024e6, c1=8400 + 16 + 512, c2=8400 + 512, bw1=512, bw2=512,
         expect=[128, 0, 3968, 128]),
    dict(fft=8192, fs=1024e6, c1=8400 + 512, c2=8400 + 16 + 512, bw1=512, bw2=512,
         expect=[-128, 128, 4096, 0]),
    dict(fft=1024, fs=32e6, c1=8400 + 16, c2=8400 + 16, bw1=16, bw2=16,
         expect=[0, 0, 512, 0]),
    dict(fft=1024, fs=32e6, c1=8400 + 16, c2=8400 + 16 + 40, bw1=16, bw2=16, expect=None),
]

delay = [
    # polynomial branch (main.rs:209-230): tau1 = 3.25e-6 s at fs = 1 MHz -> 3.25 samples
    # -> int1 = 3, frac1 = 0.25e-6; fringe -2*pi*1e5*3.25e-6 = -0.65*pi rad
    dict(cfg=dict(frame_dt=1024e-6, fs=1e6, net_d1_base=3.25e-6, lo1_hz=1e5), frame=0,
         expect=dict(int1=3, int2=0, frac1=0.25e-6, frac2=0.0,
                     fr_lo1=[-0.45399049973954675, -0.8910065241883679], fr_lo2=[1.0, 0.0])),
    # table branch (main.rs:187-208): frame 1, frame_dt 0.25 s -> t_mid 0.375 s;
    # gd = 1e-6*0.625 + 2e-6*0.375 = 1.375e-6 -> 1.375 samples -> int 1, frac 0.375e-6
    dict(cfg=dict(frame_dt=0.25, fs=1e6), table=[1e-6, 2e-6], frame=1,
         expect=dict(int1=1, int2=0, frac1=0.375e-6, frac2=0.0, fr_lo1=[1.0, 0.0],
                     fr_lo2=[1.0, 0.0])),
    # table branch with relative clock: clock2 - clock1 = 2e-6 + 0 -> 3.375 samples -> 3
    dict(cfg=dict(frame_dt=0.25, fs=1e6, clock2_delay_s=2e-6), table=[1e-6, 2e-6], frame=1,
         expect=dict(int1=3, int2=0, frac1=0.375e-6, frac2=0.0, fr_lo1=[1.0, 0.0],
                     fr_lo2=[1.0, 0.0])),
    # negative delay rounds half away from zero: -2.5 samples -> -3, frac +0.5e-6
    dict(cfg=dict(frame_dt=1024e-6, fs=1e6, net_d1_base=-2.5e-6), frame=0,
         expect=dict(int1=-3, int2=0, frac1=0.5e-6, frac2=0.0, fr_lo1=[1.0, 0.0],
                     fr_lo2=[1.0, 0.0])),
]

xcf_phase = [  # main.rs:132-149: step1 = -2 pi df frac1 = -0.2 pi, start = 2*step1
    dict(df=1e3, frac1=1e-4, frac2=0.0, a1s=2, a2s=0,
         expect=[0.30901699437494745, -0.9510565162951535, 0.8090169943749475,
                 -0.5877852522924731]),
]

quantise = [  # utils.rs:378-410: nearest level, first index wins ties, LSB-first, pad tail
    dict(samples=[-2.0, 0.1, 0.6, 5.0], bits=2, levels=L2, shuffle=IDENT,
         expect=[0xE8, 0x00, 0x00, 0x00]),
    dict(samples=[0.0], bits=2, levels=L2, shuffle=IDENT, expect=[0x01, 0x00, 0x00, 0x00]),
]

level_power = [dict(levels=L2, expect=1.25), dict(levels=[-3.0, -1.0, 1.0, 3.0], expect=5.0)]

# Known answers the reference documents itself (README.md), beside the
# hand-derived vectors above:
readme = dict(
    # README.md:225-235: n = round(tau fs), eps = tau - n/fs; "12.983 samples is
    # handled as n=13, eps=-0.017 sample", "12.345 samples ... n=12, eps=+0.345"
    delay_split=[dict(samples=12.983, fs=1e6, n=13, eps_samples=-0.017),
                 dict(samples=12.345, fs=1e6, n=12, eps_samples=0.345)],
    # README.md:241-243: "For 2-bit sampling: n=12 samples means 24 bits (3 bytes)"
    bit_offset=[dict(bits=2, samples=12, offset_bits=24, offset_bytes=3)],
    # README.md:276-293: inv = 1/(0.5 P nf fft^2), P11 = mean(level1^2),
    # P12 = sqrt(P11 P22); "typical 2-bit levels [-1.5, 0.5, -0.5, 1.5]:
    # mean(level^2) = 1.25".  fft = 8, nf = 10: inv = 1/(0.5 1.25 10 64) = 1/400
    normalize=[dict(levels=[-1.5, 0.5, -0.5, 1.5], p=1.25, fft=8, nf=10,
                    acc=[400.0, 800.0, 1200.0, 1600.0, 2000.0], expect=[1.0, 2.0, 3.0, 4.0])],
    # P12 of the typical 2-bit levels against +-1/+-3 (P22 = 5): sqrt(1.25 * 5) = 2.5
    cross_power=[dict(levels1=[-1.5, 0.5, -0.5, 1.5], levels2=[-3.0, -1.0, 1.0, 3.0], p12=2.5)],
)

normalize = [  # main.rs:2645-2683: inv = 1/(0.5*P*nf*N^2), first N/2 bins
    dict(fft=4, nf=2, p=1.25, acc=[20.0, 40.0, 60.0], expect=[1.0, 2.0]),
]

rfft = [  # unnormalised DFT (utils.rs:47-59)
    dict(n=16, kind="cos3", expect_bin=3, expect_value=[8.0, 0.0]),
    dict(n=16, kind="delta1"),
]

out = dict(decode=decode, shift=shift, parse_shuffle=parse_shuffle, band=band, delay=delay,
           xcf_phase=xcf_phase, quantise=quantise, level_power=level_power,
           normalize=normalize, rfft=rfft, readme=readme)
Path(__file__).with_name("kat.json").write_text(json.dumps(out, indent=1))
print("wrote", Path(__file__).with_name("kat.json"))
