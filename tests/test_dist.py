"""The N > 1 path of bench.py on CPU: two gloo ranks take the same collective steps (barrier,
max over ranks) and agree on the maximum; replicas exchange nothing else."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    from datetime import timedelta
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), ".."))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        bench.barrier(world)
        t = bench.max_over_ranks(10.0 + 5.0 * rank, world)
        bench.barrier(world)
        out[rank] = t
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_max_over_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(90)
        assert all(p.exitcode == 0 for p in procs)
        assert dict(out) == {0: 15.0, 1: 15.0}
