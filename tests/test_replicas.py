"""The bench's multi-GPU path is replicas only (the correlation shards by scan
or sector with no data-path collective): each rank times its own work and
the whole-job value is every rank's samples over the slowest rank's time.
Checked here with two gloo ranks on the CPU; the reference arm runs on rank 0
alone and the other ranks exit without output."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r processed (r + 1) Gsample in 10 (r + 1) ms
        v, ms = bench.replica_throughput(dist, (rank + 1) * 1e9, 10.0 * (rank + 1), "cpu")
        Path(out, f"r{rank}.json").write_text(json.dumps({"value": v, "ms": ms}))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        got = json.loads(Path(tmp_path, f"r{r}.json").read_text())
        # (1 + 2) Gsample over the slowest rank's 20 ms, the same on every rank
        assert got["ms"] == pytest.approx(20.0)
        assert got["value"] == pytest.approx(3e9 / 20e-3 / 1e9)


def test_replica_throughput_single_process():
    sys.path.insert(0, str(ROOT))
    import bench

    v, ms = bench.replica_throughput(None, 2e9, 4.0, "cpu")
    assert ms == 4.0 and v == pytest.approx(500.0)


def test_reference_arm_nonzero_rank_exits_silently():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "3"], capture_output=True, text=True,
                       env=env, timeout=120, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
