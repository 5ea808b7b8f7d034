"""The multi-GPU layout (replicas, vie_fft_b200/replicas.py) with two gloo
ranks on the CPU: each rank takes its own instances, the job time is the
slowest rank's, and throughput counts every rank's instances."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from vie_fft_b200.replicas import replica_wavelength, shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from vie_fft_b200.replicas import max_over_ranks, throughput
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard(range(11), rank, world)
        ms_local = 100.0 + 50.0 * rank          # rank 1 is the slow one
        value, ms_max = throughput(len(mine), ms_local)
        out.put((rank, mine, value, ms_max, max_over_ranks(-rank)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, v0, t0, x0), (r1, m1, v1, t1, x1) = res
    # the shards cover the batch once
    assert sorted(m0 + m1) == list(range(11)) and not set(m0) & set(m1)
    # job time = slowest rank; every rank reports the same aggregate
    assert t0 == t1 == 150.0
    assert v0 == v1 == pytest.approx(11 * 1e3 / 150.0)
    assert x0 == x1 == 0.0


def test_replica_helpers():
    assert replica_wavelength(550.0, 0) == 550.0 and replica_wavelength(550.0, 3) == 565.0
    assert shard("abcdefg", 1, 3) == ["b", "e"]
    with pytest.raises(ValueError):
        shard([1, 2], 2, 2)
