"""MSM split across ranks with the real kernels: two gloo ranks, each with its own context on
the one GPU (their kernels never wait on each other; the one-point exchange goes through host
memory), must reproduce the single-GPU MSM and, at small sizes, the oracle."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, scl, pts, ec2, out):
    import sys
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), ".."))
    from cusnarks_b200 import Context
    from cusnarks_b200.sharded import sharded_msm, shard_range
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    ctx = Context(0)
    try:
        n = scl.shape[0]
        lo, hi = shard_range(n, rank, world)
        s_t = torch.from_numpy(scl[lo:hi].view(np.int32).copy()).cuda()
        p_t = torch.from_numpy(pts[lo:hi].view(np.int32).copy()).cuda()
        res = sharded_msm(ctx, s_t, p_t, ec2=ec2)
        out[rank] = res.cpu().numpy().view(np.uint32).tolist()
    finally:
        ctx.close()
        dist.destroy_process_group()


def _run(world, scl, pts, ec2):
    mpc = mp.get_context("spawn")
    with mpc.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [mpc.Process(target=_rank, args=(r, world, port, scl, pts, ec2, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(240)
        assert all(p.exitcode == 0 for p in procs)
        return [out[r] for r in range(world)]


@pytest.mark.timeout(300)
@pytest.mark.parametrize("n,ec2", [(1 << 12, False), (777, True)])
def test_sharded_msm_two_ranks_matches_oracle(oracle, n, ec2):
    from tests.sharded_case import case
    scl, pts = case(n, ec2)
    want = np.asarray(oracle.msm(scl, pts, int(ec2))).reshape(-1).tolist()
    got = _run(2, scl, pts, ec2)
    assert got[0] == want and got[1] == want


@pytest.mark.timeout(300)
def test_sharded_msm_large_matches_single_gpu():
    import torch
    from cusnarks_b200 import Context
    from cusnarks_b200.synth import random_field, g1_generator
    n = 1 << 18
    rng = np.random.Generator(np.random.PCG64(99))
    ctx = Context(0)
    try:
        k = torch.from_numpy(random_field(rng, n).view(np.int32)).cuda()
        g = torch.from_numpy(g1_generator().view(np.int32)).cuda()
        pts = torch.empty((n, 16), dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        ctx.scmul_device(k.data_ptr(), g.data_ptr(), n, pts.data_ptr(), ec2=False, point_stride_words=0)
        ctx.sync()
        scl = random_field(rng, n)
        s_t = torch.from_numpy(scl.view(np.int32).copy()).cuda()
        single = torch.zeros(16, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        ctx.msm_device(s_t.data_ptr(), pts.data_ptr(), n, single.data_ptr())
        ctx.sync()
        want = single.cpu().numpy().view(np.uint32).tolist()
        pts_h = pts.cpu().numpy().view(np.uint32)
    finally:
        ctx.close()
    got = _run(2, np.ascontiguousarray(scl), np.ascontiguousarray(pts_h), False)
    assert got[0] == want and got[1] == want
