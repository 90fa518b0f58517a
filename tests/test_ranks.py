"""Multi-rank host logic of the replica-parallel runs on CPU (gloo, world size 2):
distinct per-rank device keys, and the job timing as max over ranks with attempts
summed over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from scemc import ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, att = ranks.aggregate(10.0 + 5.0 * rank, 100.0 * (rank + 1), dist)
        out[rank] = (ms, att, tuple(ranks.rank_keys(7, rank, 4)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation_and_keys():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        ps = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0  # slowest rank
    assert res[0][1] == res[1][1] == 300.0  # all attempts
    assert not set(res[0][2]) & set(res[1][2])
    assert ranks.aggregate(3.0, 4.0) == (3.0, 4.0)  # single process
