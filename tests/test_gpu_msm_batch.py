"""Batched MSM (one pass over many instances of uneven size): every instance's result equals
the single-instance GPU MSM with the same window and the oracle, word for word; direct runs,
the first graph capture and graph replays agree; the autotuner's windows feed the batch."""
import numpy as np
import pytest

from oracle.oracle import random_field
from tests.gpu_common import g1_generator_mont, g2_generator_mont

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from cusnarks_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _points(ctx, n, ec2, seed):
    """n bases k_i * G on the GPU (k_i seeded)."""
    import torch
    pw = 32 if ec2 else 16
    k = random_field(np.random.Generator(np.random.PCG64(seed)), n, 1)
    dk = torch.from_numpy(k.view(np.int32)).cuda()
    g = torch.from_numpy((g2_generator_mont() if ec2 else g1_generator_mont()).view(np.int32)).cuda()
    dp = torch.zeros((max(n, 1), pw), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    if n:
        ctx.scmul_device(dk.data_ptr(), g.data_ptr(), n, dp.data_ptr(), ec2=ec2, point_stride_words=0)
        ctx.sync()
    return dp


def _case(ctx, sizes, windows, ec2, seed):
    import torch
    pw = 32 if ec2 else 16
    ins = []
    for q, n in enumerate(sizes):
        s = random_field(np.random.Generator(np.random.PCG64(seed + 1000 + q)), max(n, 1), 1)
        ds = torch.from_numpy(s.view(np.int32)).cuda()
        dp = _points(ctx, n, ec2, seed + q)
        ins.append((s, ds, dp, torch.zeros(pw, dtype=torch.int32, device="cuda")))
    torch.cuda.synchronize()
    jobs = [(ds.data_ptr(), dp.data_ptr(), n, do.data_ptr(), w)
            for (s, ds, dp, do), n, w in zip(ins, sizes, windows)]
    return ins, jobs


def _single(ctx, ds, dp, n, w, ec2):
    import torch
    out = torch.zeros(32 if ec2 else 16, dtype=torch.int32, device="cuda")
    ctx.msm_device(ds.data_ptr(), dp.data_ptr(), n, out.data_ptr(), ec2=ec2, window=w)
    ctx.sync()
    return out.cpu().numpy().view(np.uint32).copy()


@pytest.mark.parametrize("task", [0, 8, 64])
@pytest.mark.parametrize("ec2", [False, True])
def test_batch_equals_single_and_oracle(ctx, oracle, ec2, task):
    """task 0: the tile the batch's size picks (8 here: small instances); 8: buckets split
    into many partial sums; 64: few splits."""
    sizes = [0, 1, 3, 100, 1000, 2048, 1 << 13, 1 << 15] if not ec2 else [5, 0, 300, 2048, 1 << 12]
    windows = [0, 0, 5, 0, 9, 0, 12, 0] if not ec2 else [0, 7, 0, 11, 0]
    ins, jobs = _case(ctx, sizes, windows, ec2, seed=7 if ec2 else 3)
    batch = ctx.msm_batch(jobs, ec2=ec2, task=task)
    try:
        got = []
        for mode in (False, True, True):          # direct, capture + launch, replay
            for (_, _, _, do) in ins:
                do.zero_()
            import torch
            torch.cuda.synchronize()
            batch.run(graph=mode)
            ctx.sync()
            got.append([do.cpu().numpy().view(np.uint32).copy() for (_, _, _, do) in ins])
        wins = batch.windows()
        for q, n in enumerate(sizes):
            want = _single(ctx, ins[q][1], ins[q][2], n, wins[q], ec2)
            for g in got:
                assert np.array_equal(g[q], want), (q, n)
            if 0 < n <= 2048:
                p = ins[q][2].cpu().numpy().view(np.uint32)[:n]
                assert np.array_equal(want, oracle.msm(ins[q][0][:n], p, ec2=1 if ec2 else 0)), (q, n)
        for q, w in enumerate(windows):
            if w:
                assert wins[q] == w, q
    finally:
        batch.close()


def test_autotune_feeds_batch(ctx):
    tuned = ctx.msm_autotune(10, 12)
    assert len(tuned) == 3 and all(4 <= w <= 22 for w in tuned)
    assert [ctx.msm_tuned_window(1 << L) for L in (10, 11, 12)] == tuned
    sizes = [1 << 10, 1 << 11, 1 << 12, 1500]
    ins, jobs = _case(ctx, sizes, [0] * 4, False, seed=21)
    batch = ctx.msm_batch(jobs)
    try:
        assert batch.windows()[:3] == tuned and batch.windows()[3] == tuned[1]
        batch.run(graph=True)
        ctx.sync()
        for q, n in enumerate(sizes):
            got = ins[q][3].cpu().numpy().view(np.uint32)
            assert np.array_equal(got, _single(ctx, ins[q][1], ins[q][2], n, 0, False)), q
    finally:
        batch.close()


@pytest.mark.parametrize("ec2", [False, True])
def test_batch_config4_sizes_against_oracle(ctx, oracle, ec2):
    """Instances of the batched configuration's size range up to 2^16 terms (log-uniform and
    ragged), one batch, graph replay: every instance equals the oracle's multi-exp."""
    import torch
    if ec2:
        sizes = [1 << 10, 1 << 16, 5000, 1 << 13]
    else:
        sizes = [1 << 16, 1 << 10, 1 << 11, 1 << 12, 1 << 13, 1 << 14, 1 << 15, 3000, 50000]
    ins, jobs = _case(ctx, sizes, [0] * len(sizes), ec2, seed=90 if ec2 else 80)
    batch = ctx.msm_batch(jobs, ec2=ec2)
    try:
        batch.run(graph=True)
        ctx.sync()
        for (_, _, _, do) in ins:
            do.zero_()
        torch.cuda.synchronize()
        batch.run(graph=True)  # replay
        ctx.sync()
        for q, n in enumerate(sizes):
            got = ins[q][3].cpu().numpy().view(np.uint32)
            p = ins[q][2].cpu().numpy().view(np.uint32)[:n]
            assert np.array_equal(got, oracle.msm(ins[q][0][:n], p, ec2=1 if ec2 else 0)), (q, n)
    finally:
        batch.close()
