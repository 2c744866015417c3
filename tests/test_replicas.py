"""The multi-GPU path is replicas: events shard by rank with no exchange, and
the job's rate is all ranks' events over the slowest rank's time.  Checked
here with two gloo ranks on the CPU (pixeltrack-standalone_b200/replicas.py,
the helpers bench.py uses under torchrun)."""
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "pixeltrack-standalone_b200")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, ms, q):
    sys.path.insert(0, PKG)
    import datetime
    import torch.distributed as dist
    import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        seeds = replicas.shard_seeds(rank, world, 4, 1000)
        rate, worst = replicas.job_rate(640, ms[rank])
        q.put((rank, seeds, rate, worst))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ms = [100.0, 160.0]  # rank 1 is the slower
    procs = [ctx.Process(target=_rank, args=(r, 2, port, ms, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, rate0, w0), (r1, s1, rate1, w1) = out
    assert set(s0).isdisjoint(s1) and len(s0) == len(s1) == 4
    assert w0 == w1 == 160.0
    assert rate0 == rate1 == pytest.approx(2 * 640 / 0.160)


def test_single_process_is_local():
    sys.path.insert(0, PKG)
    import replicas
    assert replicas.job_rate(100, 50.0) == (2000.0, 50.0)
    assert replicas.shard_seeds(0, 1, 3, 7) == [7, 8, 9]
    with pytest.raises(ValueError):
        replicas.shard_seeds(2, 2, 3, 7)
