"""bench.py's multi-GPU bookkeeping with two ranks on CPU (gloo): replicas take
disjoint states, the job time is the slowest rank's, and the aggregate counts
every rank's states.  No GPU and no collective on the data path."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 * (rank + 1), world, "cpu")
        out[rank] = (ms, bench.rank_seeds(rank, 20), bench.job_states(12, world))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == pytest.approx(20.0)
    assert not set(res[0][1]) & set(res[1][1])
    assert res[0][2] == res[1][2] == 24
