"""MSM split across ranks (cusnarks_b200.sharded) on CPU: gloo ranks, with the oracle standing
in for each rank's device MSM and point sum, must give the single-MSM result on every rank."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cusnarks_b200.sharded import shard_range


def test_shard_range_covers_terms():
    for n in (0, 1, 5, 16, 1000, 1 << 20):
        for world in (1, 2, 3, 8):
            rs = [shard_range(n, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            sizes = [hi - lo for lo, hi in rs]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


class _OracleCtx:
    """Host stand-in with the Context calls sharded_msm makes (CPU tensors, raw pointers)."""

    def __init__(self):
        from oracle.oracle import Oracle
        self.o = Oracle()

    @staticmethod
    def _view(ptr, words):
        return np.ctypeslib.as_array((ctypes.c_uint32 * words).from_address(ptr))

    def msm_device(self, ds, dp, n, dout, ec2=False, window=0):
        pw = 32 if ec2 else 16
        s = self._view(ds, 8 * n).reshape(n, 8).copy()
        p = self._view(dp, pw * n).reshape(n, pw).copy()
        self._view(dout, pw)[:] = np.asarray(self.o.msm(s, p, int(ec2))).reshape(-1)

    def point_sum_device(self, dp, n, dout, ec2=False, dims=2):
        pw = 32 if ec2 else 16
        p = self._view(dp, pw * n).reshape(n, pw).copy()
        ones = np.zeros((n, 8), np.uint32)
        ones[:, 0] = 1
        self._view(dout, pw)[:] = np.asarray(self.o.msm(ones, p, int(ec2))).reshape(-1)

    def sync(self):
        pass


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, n, ec2, out):
    import sys
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), ".."))
    from cusnarks_b200.sharded import sharded_msm, shard_range
    from tests.sharded_case import case
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        scl, pts = case(n, ec2)
        lo, hi = shard_range(n, rank, world)
        s_t = torch.from_numpy(scl[lo:hi].view(np.int32).copy())
        p_t = torch.from_numpy(pts[lo:hi].view(np.int32).copy())
        res = sharded_msm(_OracleCtx(), s_t, p_t, ec2=ec2)
        out[rank] = res.numpy().view(np.uint32).tolist()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
@pytest.mark.parametrize("world,n,ec2", [(2, 40, False), (3, 7, False), (2, 12, True), (4, 3, False)])
def test_sharded_msm_equals_single(world, n, ec2):
    from oracle.oracle import Oracle
    from tests.sharded_case import case
    scl, pts = case(n, ec2)
    want = np.asarray(Oracle().msm(scl, pts, int(ec2))).reshape(-1).tolist()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, n, ec2, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(150)
        assert all(p.exitcode == 0 for p in procs)
        assert all(out[r] == want for r in range(world))
