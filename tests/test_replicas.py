"""Replica path of multi-GPU runs on CPU: two gloo ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from energy_level_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r "took" 1 + r seconds and processed 3 units
        elapsed, other = replicas.max_over_ranks([1.0 + rank, 10.0 - rank], dist)
        rate = replicas.aggregate_rate(3, world, elapsed)
        out.put((rank, elapsed, other, rate, replicas.replica_seed(2, rank)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, elapsed, other, rate, seed in res:
        assert elapsed == 2.0 and other == 10.0
        assert rate == pytest.approx(3.0)
    assert res[0][4] == 2 and res[1][4] == 1002


def test_single_process_is_identity():
    assert replicas.max_over_ranks([1.5, 2.5]) == [1.5, 2.5]
    assert replicas.aggregate_rate(5, 1, 2.0) == 2.5
    with pytest.raises(ValueError):
        replicas.aggregate_rate(1, 1, 0.0)
