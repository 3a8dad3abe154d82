"""Batched sectors of many scans (fxc_batch_*), called through the C ABI:
every sector of a mixed batch (FFT 1024-16384, 1/2/4/8-bit stations,
shuffles, LSB, both output grids, uneven frame counts) within the stated
tolerance of the FP64 oracle and of the per-scan path; a sector's products
identical bit for bit alone and in any mix, with and without CUDA graphs;
sectors the batch kernels do not cover taken by the per-scan path; the
autotuner's shapes; argument errors."""
import numpy as np
import pytest

import oracle
from _cases import (assert_sector_close, assert_spectra_close, make_scan, signal_raw,
                    spectral_errors, to_fxc)

pytestmark = pytest.mark.gpu

DELAY = dict(net_d1_base=3.3e-7, total_rate1_base=2.1e-6, lo1_hz=8.4e9, lo2_hz=8.4e9)

# (scan kwargs, frames): every batch group, bit depth, shuffle kind and grid
MIX = [
    (dict(fft=1024, bits1=2, bits2=2, shuffle="generic", band=(8, 0, 504, 8)), 700),
    (dict(fft=1024, bits1=1, bits2=4, shuffle="pairswap", lsb2=True, band=(0, 0, 512, 0),
          grid=1), 131),
    (dict(fft=2048, bits1=2, bits2=2, shuffle="sample2", lsb1=True, band=(-16, 16, 1024, 0)),
     333),
    (dict(fft=2048, bits1=8, bits2=8, shuffle="generic", band=(4, 0, 1020, 4), grid=1), 65),
    (dict(fft=4096, bits1=2, bits2=2, band=(40, 0, 2008, 40)), 517),
    (dict(fft=4096, bits1=4, bits2=2, shuffle="generic", lsb1=True, lsb2=True,
          band=(0, 0, 2048, 0)), 3),
    (dict(fft=8192, bits1=2, bits2=2, shuffle="generic", lsb1=True, band=(64, 0, 4032, 64)),
     611),
    (dict(fft=8192, bits1=1, bits2=2, shuffle="pairswap", band=(-40, 40, 4096, 0), grid=1), 1),
    (dict(fft=8192, bits1=8, bits2=4, shuffle="generic", band=(0, 0, 4096, 0),
          products=oracle.PROD_ACF | oracle.PROD_ACF_OVERLAP_ONLY | oracle.PROD_XCF), 90),
    (dict(fft=16384, bits1=2, bits2=2, shuffle="generic", band=(128, 0, 8064, 128)), 200),
    (dict(fft=16384, bits1=4, bits2=1, lsb2=True, band=(-64, 64, 8192, 0), grid=1), 37),
]


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def build(engine, cases, seed0=0):
    out = []
    for k, (kw, nf) in enumerate(cases):
        scan = make_scan(delay=DELAY, fs=512e6, seed=k, **kw)
        if nf:
            r1, r2 = signal_raw(scan, nf, seed=seed0 + 100 + k, rho=0.2, delay_samples=6.4)
        else:  # an empty sector still takes 16-byte aligned buffers
            r1, r2 = np.zeros(16, np.uint8), np.zeros(16, np.uint8)
        out.append(dict(scan=scan, nf=nf, r1=r1, r2=r2, d1=dev(r1), d2=dev(r2),
                        first=7 * k + 1, s=engine.open_scan(to_fxc(scan))))
    return out


def run(batch, items):
    import torch

    accs = [torch.empty(5 * it["scan"].h, dtype=torch.float64, device="cuda") for it in items]
    batch.run_device([it["s"] for it in items], [it["d1"] for it in items],
                     [it["d2"] for it in items], [it["nf"] for it in items],
                     [it["first"] for it in items], accs)
    torch.cuda.synchronize()
    for it in items:
        it["s"].check()
    res = []
    for it, a in zip(items, accs):
        h = it["scan"].h
        a = a.cpu().numpy()
        res.append(dict(acf11=a[:h], acf22=a[h:2 * h], xcf=a[2 * h:4 * h].view(np.complex128),
                        phased=a[4 * h:]))
    return res


def close(items):
    for it in items:
        it["s"].close()


@pytest.fixture(scope="module")
def mix(engine):
    items = build(engine, MIX)
    yield items
    close(items)


def same(a, b):
    return all(np.array_equal(a[k], b[k]) for k in ("acf11", "acf22", "xcf", "phased"))


def test_batch_mix_vs_fp64_and_scan_path(fxc_lib, engine, mix):
    b = fxc_lib.Batch(engine)
    got = run(b, mix)
    for it, g in zip(mix, got):
        scan, nf = it["scan"], it["nf"]
        ref = oracle.fp64_sector_corr(scan, it["r1"], it["r2"], nf, first_frame=it["first"])
        ref_acf = ref
        if scan.products & oracle.PROD_ACF_OVERLAP_ONLY:
            import dataclasses
            full = dataclasses.replace(scan, products=oracle.PROD_ACF)
            ref_acf = oracle.fp64_sector_corr(full, it["r1"], it["r2"], nf, first_frame=it["first"])
        assert_sector_close(g, ref, scan, f"batch fft={scan.fft} nf={nf}", nf=nf, ref_acf=ref_acf)
        one = it["s"].sector_device(it["d1"], it["d2"], nf, first_frame=it["first"])
        for k in ("acf11", "acf22"):
            if np.any(one[k]):
                rel, ph, ab = spectral_errors(g[k], one[k])
                assert ab < 2e-6, (scan.fft, k, ab)
        assert np.all(g["phased"] == 0)
    # 2 + one kernel per FFT length present
    assert b.launches() == 2 + 5
    b.close()


def test_batch_alone_equals_mix_and_graphs(fxc_lib, engine, mix):
    plain = fxc_lib.Batch(engine)
    graph = fxc_lib.Batch(engine, use_graphs=True)
    both = run(plain, mix)
    g1 = run(graph, mix)
    g2 = run(graph, mix)  # replay
    for k, it in enumerate(mix):
        alone = run(plain, [it])[0]
        assert same(alone, both[k]), (k, it["scan"].fft)
        assert same(g1[k], both[k]) and same(g2[k], both[k]), k
    # another batch of the same FFT lengths replays the same graph with new counts
    sub = [mix[0], mix[2], mix[4], mix[6], mix[9]]
    g3 = run(graph, sub[::-1])[::-1]
    for it, r in zip(sub, g3):
        assert same(r, both[mix.index(it)])
    plain.close()
    graph.close()


def test_batch_fallback_sectors(fxc_lib, engine):
    """Phased products, FFT 32768, an odd band shift at 16384 and an empty
    sector take the per-scan path inside the same call."""
    cases = [
        (dict(fft=32768, band=(256, 0, 16128, 256)), 20),
        (dict(fft=16384, band=(3, 0, 8189, 3)), 30),
        (dict(fft=4096, products=oracle.PROD_ACF | oracle.PROD_XCF | oracle.PROD_PHASED,
              band=(0, 0, 2048, 0)), 50),
        (dict(fft=2048, band=(0, 0, 1024, 0)), 0),
        (dict(fft=8192, band=(0, 0, 4096, 0)), 40),
    ]
    items = build(engine, cases, seed0=50)
    b = fxc_lib.Batch(engine)
    got = run(b, items)
    for it, g in zip(items, got):
        one = it["s"].sector_device(it["d1"], it["d2"], it["nf"], first_frame=it["first"])
        if it["nf"] == 0:
            assert all(np.all(g[k] == 0) for k in ("acf11", "acf22", "xcf", "phased"))
            continue
        if it["scan"].fft == 8192:
            ref = oracle.fp64_sector_corr(it["scan"], it["r1"], it["r2"], it["nf"],
                                          first_frame=it["first"])
            assert_sector_close(g, ref, it["scan"], "batched 8192", nf=it["nf"], ref_acf=ref)
        else:  # the per-scan path itself
            assert same(g, one), it["scan"].fft
    b.close()
    close(items)


def test_batch_autotune_shapes(fxc_lib, engine):
    b = fxc_lib.Batch(engine, autotune=True)
    items = build(engine, [(dict(fft=1024, band=(0, 0, 512, 0)), 400),
                           (dict(fft=8192, band=(0, 0, 4096, 0)), 300)], seed0=90)
    got = run(b, items)  # tunes 1024 and 8192 at first use
    for fft in (1024, 8192):
        sh = b.shape(fft)
        assert sh["gsps"] > 0 and sh["ctas_per_sm"] >= 1
        assert sh["item_frames"] in (32, 64, 128, 256, 512)
        assert sh["fpc"] in ((1, 2, 4) if fft == 1024 else (1,))
    assert b.shape(2048)["gsps"] == 0  # not tuned yet
    b.autotune(2048)
    assert b.shape(2048)["gsps"] > 0
    for it, g in zip(items, got):
        ref = oracle.fp64_sector_corr(it["scan"], it["r1"], it["r2"], it["nf"],
                                      first_frame=it["first"])
        assert_sector_close(g, ref, it["scan"], f"tuned {it['scan'].fft}", nf=it["nf"],
                            ref_acf=ref)
    b.close()
    close(items)


@pytest.mark.parametrize("fpc_fft", [1024, 2048, 4096])
def test_batch_variants_agree(fxc_lib, engine, fpc_fft):
    """Every frames-per-iteration variant agrees with the others and with the
    FP64 oracle (the per-frame FFT and the 32-frame f32 flush groups are the
    same; the bins a thread owns, hence the fringe-ramp recurrence steps,
    differ, so agreement is to FP32 rounding, not bit for bit)."""
    items = build(engine, [(dict(fft=fpc_fft, band=(0, 0, fpc_fft // 2, 0)), 257),
                           (dict(fft=fpc_fft, bits1=4, shuffle="generic",
                                 band=(8, 0, fpc_fft // 2 - 8, 8), grid=1), 96)], seed0=70)
    b = fxc_lib.Batch(engine, item_frames=64)
    base = run(b, items)
    for fpc in ((1, 2, 4) if fpc_fft < 4096 else (1, 2)):
        b.set_shape(fpc_fft, fpc, 64)
        assert b.shape(fpc_fft)["fpc"] == fpc
        got = run(b, items)
        for it, g, r in zip(items, got, base):
            for k in ("acf11", "acf22"):
                assert spectral_errors(g[k], r[k])[2] < 1e-6, (fpc_fft, fpc, k)
            ref = oracle.fp64_sector_corr(it["scan"], it["r1"], it["r2"], it["nf"],
                                          first_frame=it["first"])
            assert_sector_close(g, ref, it["scan"], f"fpc={fpc} fft={fpc_fft}", nf=it["nf"],
                                ref_acf=ref)
    with pytest.raises(fxc_lib.FxcError):
        b.set_shape(fpc_fft, 3, 64)
    with pytest.raises(fxc_lib.FxcError):
        b.set_shape(fpc_fft, 1, 48)
    b.close()
    close(items)


def test_batch_errors(fxc_lib, engine, mix):
    import torch

    b = fxc_lib.Batch(engine)
    it = mix[0]
    acc = torch.empty(5 * it["scan"].h, dtype=torch.float64, device="cuda")
    with pytest.raises(fxc_lib.FxcError) as e:
        b.run_device([it["s"], it["s"]], [it["d1"]] * 2, [it["d2"]] * 2, [10, 10], [0, 0],
                     [acc, acc])
    assert e.value.status == fxc_lib.EINVAL
    other = fxc_lib.Engine(0)
    s2 = other.open_scan(to_fxc(it["scan"]))
    with pytest.raises(fxc_lib.FxcError) as e:
        b.run_device([s2], [it["d1"]], [it["d2"]], [10], [0], [acc])
    assert e.value.status == fxc_lib.EINVAL
    with pytest.raises(fxc_lib.FxcError) as e:
        b.autotune(65536)
    assert e.value.status == fxc_lib.EUNSUPPORTED
    s2.close()
    other.close()
    b.close()


PHASED = oracle.PROD_PHASED | oracle.PROD_RAW
PH_MIX = [
    (dict(fft=1024, bits1=2, bits2=2, shuffle="generic", lsb1=True, band=(8, 0, 504, 8),
          products=PHASED), 300),
    (dict(fft=2048, bits1=1, bits2=4, shuffle="pairswap", band=(-16, 16, 1024, 0), grid=1,
          products=PHASED, w1=0.7, w2=1.3), 77),
    (dict(fft=4096, bits1=2, bits2=2, lsb1=True, lsb2=True, band=(40, 0, 2008, 40),
          products=PHASED), 129),
    (dict(fft=8192, bits1=2, bits2=8, shuffle="generic", band=(64, 0, 4032, 64),
          products=PHASED), 95),
    (dict(fft=8192, bits1=2, bits2=2, band=(0, 0, 4096, 0), products=oracle.PROD_PHASED), 40),
    # FFT 16384 with 2-bit stations: the two-row kernel's batch group
    (dict(fft=16384, bits1=2, bits2=2, band=(128, 0, 8064, 128), products=PHASED), 9),
    # the same group's wide layout (a 4-bit station)
    (dict(fft=16384, bits1=4, bits2=2, band=(0, 0, 8192, 0), products=PHASED), 5),
    # per-scan path inside the same call: phased above FFT 16384
    (dict(fft=32768, bits1=2, bits2=2, band=(0, 0, 16384, 0), products=PHASED), 4),
    # a correlation sector beside them
    (dict(fft=4096, bits1=2, bits2=2, shuffle="generic", band=(40, 0, 2008, 40)), 200),
]


def run_raw(batch, items):
    import torch

    accs = [torch.empty(5 * it["scan"].h, dtype=torch.float64, device="cuda") for it in items]
    raws = [torch.full((max(1, it["nf"] * it["scan"].bpf(it["scan"].bits_out)),), 0xA5,
                       dtype=torch.uint8, device="cuda")
            if it["scan"].products & oracle.PROD_RAW else None for it in items]
    batch.run_device_raw([it["s"] for it in items], [it["d1"] for it in items],
                         [it["d2"] for it in items], [it["nf"] for it in items],
                         [it["first"] for it in items], accs, raws)
    torch.cuda.synchronize()
    out = []
    for it, a, r in zip(items, accs, raws):
        it["s"].check()
        h = it["scan"].h
        a = a.cpu().numpy()
        d = dict(acf11=a[:h], acf22=a[h:2 * h], xcf=a[2 * h:4 * h].view(np.complex128),
                 phased=a[4 * h:])
        if r is not None:
            d["raw"] = r.cpu().numpy()[: it["nf"] * it["scan"].bpf(it["scan"].bits_out)]
        out.append(d)
    return out


def test_batch_phased_sectors(fxc_lib, engine):
    """yi-phasedarray sectors in the phased batch kernels: .raw frames equal
    the per-scan path's byte for byte, the phased power within the FP32
    tolerance of it (and of the FP64 oracle), correlation columns zero; each
    sector's products identical alone and in the mix, with graphs or not."""
    items = build(engine, PH_MIX, seed0=300)
    b = fxc_lib.Batch(engine)
    got = run_raw(b, items)
    for it, g in zip(items, got):
        sc = it["scan"]
        one = it["s"].sector_device(it["d1"], it["d2"], it["nf"], first_frame=it["first"])
        if sc.products & oracle.PROD_RAW:
            assert np.array_equal(g["raw"], one["raw"]), sc.fft
        if sc.products & oracle.PROD_PHASED:
            assert_spectra_close(g["phased"], one["phased"], f"batched phased {sc.fft}")
            assert all(np.all(g[k] == 0) for k in ("acf11", "acf22", "xcf"))
            if sc.fft <= 4096:
                ref = oracle.fp64_sector_phased(sc, it["r1"], it["r2"], it["nf"],
                                                first_frame=it["first"])
                assert_spectra_close(g["phased"], ref["phased"], f"phased vs fp64 {sc.fft}")
        else:
            for k in ("acf11", "acf22", "xcf"):
                assert_spectra_close(g[k], one[k], f"correlation beside phased {k}")
    # alone == in the mix, and graph replay
    bg = fxc_lib.Batch(engine, use_graphs=True)
    for k in range(len(items)):
        alone = run_raw(fxc_lib.Batch(engine), [items[k]])[0]
        for key in ("acf11", "acf22", "xcf", "phased"):
            assert np.array_equal(alone[key], got[k][key]), (k, key)
        if "raw" in alone:
            assert np.array_equal(alone["raw"], got[k]["raw"])
    for _ in range(2):
        again = run_raw(bg, items)
        for g0, g1 in zip(got, again):
            for key in g0:
                assert np.array_equal(g0[key], g1[key]), key
    bg.close()
    b.close()
    close(items)


PH16_MIX = [
    (dict(fft=16384, bits1=2, bits2=2, shuffle="generic", lsb1=True, band=(-64, 64, 8128, 0),
          products=PHASED), 3200),
    (dict(fft=16384, bits1=1, bits2=2, shuffle="pairswap", band=(96, 0, 8096, 96), grid=1,
          products=PHASED, w1=0.6, w2=1.4), 2900),
    (dict(fft=16384, bits1=4, bits2=4, shuffle="generic", band=(0, 0, 8192, 0),
          products=PHASED), 1500),
]


def test_batch_phased_16384_spans(fxc_lib, engine):
    """FFT-16384 phased sectors in the two-row kernel's persistent batch group,
    cut into 32-frame items: three sectors (1-, 2- and 4-bit stations, the
    last in the wide layout) give more items than resident CTAs, so CTAs run
    spans of several scans and both layouts back to back on one staging
    barrier.
    .raw frames equal the per-scan kernel's byte for byte, the phased power
    is within the FP32 tolerance of it, and the call is three launches (frame
    records, the group's kernel, the reduction)."""
    import torch

    items = build(engine, PH16_MIX, seed0=500)
    b = fxc_lib.Batch(engine, item_frames=32)
    n0 = b.launches()
    got = run_raw(b, items)
    assert b.launches() - n0 == 3
    # one 512-thread CTA per SM (the two rows fill shared memory): more items than CTAs
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert sum(-(-it["nf"] // 32) for it in items) > sms
    for it, g in zip(items, got):
        one = it["s"].sector_device(it["d1"], it["d2"], it["nf"], first_frame=it["first"])
        assert np.array_equal(g["raw"], one["raw"])
        assert_spectra_close(g["phased"], one["phased"], "batched phased 16384")
        assert all(np.all(g[k] == 0) for k in ("acf11", "acf22", "xcf"))
    b.close()
    close(items)
