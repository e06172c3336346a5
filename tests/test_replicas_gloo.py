"""The replica bookkeeping of multi-GPU runs, on CPU with gloo and world size 2."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from microcosmos_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        t, u = replicas.job_totals(10.0 + 5.0 * rank, 1000.0 * (rank + 1))
        out[rank] = (t, u, replicas.replica_seed(0, rank))
    finally:
        dist.destroy_process_group()


def test_job_totals_are_max_time_and_summed_work():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    assert res[0][:2] == res[1][:2] == (15.0, 3000.0)
    assert res[0][2] != res[1][2]


def test_job_totals_without_a_group_are_local():
    assert replicas.job_totals(3.0, 7.0) == (3.0, 7.0)
