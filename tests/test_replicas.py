"""Replica aggregation over a 2-rank gloo process group on the CPU (the same
calls bench.py makes over NCCL with one GPU per rank)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world_size, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=datetime.timedelta(seconds=60))
    try:
        from sphgpu.replicas import aggregate, share
        ms, units = aggregate(10.0 + 5.0 * rank, 1000.0 * (rank + 1))
        items = share(range(11), rank, world_size)
        out.put((rank, ms, units, items))
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation_sums_units_and_takes_the_max_time():
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
    for rank, ms, units, _ in res:
        assert ms == 15.0
        assert units == 3000.0
    shares = [r[3] for r in res]
    assert sorted(shares[0] + shares[1]) == list(range(11))
    assert not set(shares[0]) & set(shares[1])


def test_single_process_aggregation_is_the_identity():
    from sphgpu.replicas import aggregate, share
    assert aggregate(3.5, 42) == (3.5, 42.0)
    assert share([1, 2, 3], 0, 1) == [1, 2, 3]
    with pytest.raises(ValueError):
        share([1], 2, 2)
