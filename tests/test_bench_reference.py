"""The benchmark's reference arm on the CPU: it times the C restatement of the
reference path alone (the product package and its library are never loaded
in that process), on the same scan configuration as the GPU arm."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

PROBE = r"""
import json, sys
sys.path.insert(0, {root!r})
import bench
line = bench.reference_line(steps=1, warmup=1, world=1, sectors=2, nfs=64, threads=2)
maps = open("/proc/self/maps").read()
print(json.dumps(dict(line=line, fxc_module="fxc" in sys.modules,
                      libfxc_mapped="libfxc.so" in maps,
                      oracle_mapped="libfxc_oracle.so" in maps)))
"""


def test_reference_arm_loads_no_product_code():
    r = subprocess.run([sys.executable, "-c", PROBE.format(root=str(ROOT))], capture_output=True,
                       text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert not out["fxc_module"] and not out["libfxc_mapped"]
    assert out["oracle_mapped"]
    line = out["line"]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["config"]["sectors"] == 2 and line["config"]["frames_per_sector"] == 64


def test_both_arms_resolve_the_same_scan(fxc_lib, oracle_lib):
    sys.path.insert(0, str(ROOT))
    import bench

    a = bench.scan_fields(fxc_lib.band_alignment)
    b = bench.scan_fields(oracle_lib.c_band_alignment)
    assert a["band"] == b["band"] == (-128, 128, 4096, 0) or a["band"] == b["band"]
    for k in a:
        if k == "geom_table":
            assert (a[k] == b[k]).all()
        else:
            assert a[k] == b[k], k
    # the 16 MHz offset of the workload: a 128-bin shift, grid on station 1
    assert abs(a["band"][0]) == 128 and a["grid"] == 0
