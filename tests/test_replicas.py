"""The multi-GPU path is replicas only (the density path does not shard): these
CPU tests run bench.py's replica logic on two gloo ranks -- the max-over-ranks
clock, the whole-job value, and the reference arm's non-zero ranks exiting
without work."""
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


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = [30.0, 45.0][rank]                 # rank 1 is the slow replica
        t_max = bench._max_over_ranks(local_ms, dist, device="cpu")
        value = bench._replica_value(4096 * 20, world, t_max / 1000.0)
        dist.barrier()
        out.put((rank, t_max, value))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_clock():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t_max, value in got:
        assert t_max == 45.0
        assert value == pytest.approx(2 * 4096 * 20 / 0.045)


def test_single_rank_value_is_the_local_one():
    sys.path.insert(0, ROOT)
    import bench
    assert bench._max_over_ranks(12.5) == 12.5
    assert bench._replica_value(100, 1, 0.5) == 200.0


def test_reference_arm_nonzero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
