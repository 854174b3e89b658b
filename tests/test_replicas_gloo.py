"""Multi-rank host logic of bench.py (replicas only, no data-path
collective) on CPU with the gloo backend, world size 2."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    local_ms = 100.0 + 50.0 * rank            # rank 1 is the slow one
    ms = bench.slowest(local_ms, dist, "cpu")
    out[rank] = (bench.replica_seed(100, rank), ms, bench.whole_job_rate(250000, 3, world, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] != res[1][0]                       # distinct realisations
    assert res[0][1] == res[1][1] == 150.0              # max over ranks
    assert res[0][2] == pytest.approx(250000 * 3 * 2 / 0.150)
