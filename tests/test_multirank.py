"""Replicas on several ranks (bench.py --gpus N under torchrun): the timing
is the slowest rank's, the throughput counts every rank's particles, and the
reference arm prints from rank 0 only.  Run as two gloo ranks on the CPU."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = 10.0 + 7.5 * rank  # per-rank timed region, ms
        ms = bench.max_over_ranks(mine, dist)
        q.put((rank, ms, bench.replica_rate(1000, world, 4, ms)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate in res:
        assert ms == pytest.approx(17.5)  # every rank sees the slowest rank's time
        assert rate == pytest.approx(1000 * 2 * 4 / 17.5e-3)


def test_reference_arm_prints_on_rank0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                          "--steps", "1", "--warmup", "3"], capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0
    assert out.stdout.strip() == ""


def test_replica_rate_counts_every_rank():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_rate(16_777_216, 8, 10, 405.0) == pytest.approx(16_777_216 * 8 * 10 / 0.405)
    assert bench.max_over_ranks(3.25, None) == 3.25
