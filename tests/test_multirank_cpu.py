"""The bench's multi-rank plumbing on CPU (gloo, world size 2): the job's step time is the slowest
rank's, and every rank learns it. Image pairs are independent, so this reduction is the only
collective the multi-GPU run has."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    out[rank] = bench.max_over_ranks(1.5 + rank)
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(out) == {0: 2.5, 1: 2.5}


def test_max_over_ranks_alone():
    import bench
    assert bench.max_over_ranks(3.25) == 3.25
