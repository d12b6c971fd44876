"""Multi-process logic of bench.py on CPU (gloo, world size 2): independent
replicas with no collective on the data path; the only collective is the MAX
of the ranks' timings, and the whole-job rate counts every rank's bonds over
the slowest rank's time. The reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [12.5, 20.0][rank]
        ms = bench.max_over_ranks(local_ms, dist)
        out[rank] = (ms, bench.replica_rate(1000, 10, world, ms / 1e3))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_rate_gloo():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == out[1]
    ms, rate = out[0]
    assert ms == 20.0
    assert rate == pytest.approx(1000 * 10 * 2 / 0.02)


def test_single_process_is_identity():
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.replica_rate(10, 5, 1, 2.0) == 25.0


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(_free_port()))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
