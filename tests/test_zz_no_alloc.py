"""The allocation-free G1 multi-exponentiation entry point (cs_msm_g1_noalloc).

It exists for callers that may not call cudaMalloc (their device memory belongs to a
host framework's pool, or the allocation's implicit synchronisation is not acceptable on
their path).  Its scratch is a fixed device array shared by all calls, so this test
checks two consecutive calls against the regular entry point, word for word, and that a
size beyond the array is refused with an error instead of running; the smaller call is
also checked against the oracle's multi-exponentiation.  The file sorts last
so that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from cusnarks_b200.synth import random_field

pytestmark = pytest.mark.gpu


def _points(ctx, rng, n):
    import torch
    from cusnarks_b200.synth import g1_generator
    k = torch.from_numpy(random_field(rng, n).view(np.int32)).cuda()
    g = torch.from_numpy(g1_generator().view(np.int32)).cuda()
    p = torch.empty((n, 16), dtype=torch.int32, device="cuda")
    ctx.scmul_device(k.data_ptr(), g.data_ptr(), n, p.data_ptr(), point_stride_words=0)
    ctx.sync()
    return p


def test_noalloc_matches_allocating_entry_point_twice(oracle):
    import torch
    from cusnarks_b200 import Context, lib
    L = lib()
    assert L.cs_msm_noalloc_scratch_bytes() == 32 << 20
    nmax = L.cs_msm_g1_noalloc_max_terms()
    assert nmax >= 1 << 16
    ctx = Context(0)
    rng = np.random.Generator(np.random.PCG64(4242))
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for n in (1 << 16, 3000):  # two calls in a row: full size, then a smaller one
        pts = _points(ctx, rng, n)
        s = torch.from_numpy(random_field(rng, n).view(np.int32)).cuda()
        want = torch.zeros(16, dtype=torch.int32, device="cuda")
        got = torch.zeros(16, dtype=torch.int32, device="cuda")
        ctx.msm_device(s.data_ptr(), pts.data_ptr(), n, want.data_ptr())
        ctx.sync()
        torch.cuda.synchronize()
        rc = L.cs_msm_g1_noalloc(ctypes.c_void_p(s.data_ptr()), ctypes.c_void_p(pts.data_ptr()), n,
                                 ctypes.c_void_p(got.data_ptr()), ctypes.c_void_p(stream))
        assert rc == 0, L.cs_msm_g1_noalloc_error()
        torch.cuda.synchronize()
        results.append(got.cpu().numpy())
        assert np.array_equal(got.cpu().numpy(), want.cpu().numpy()), n
        if n <= 3000:  # and the oracle's multi-exp (the reference's ec_jacreduce_server_h restated)
            host = got.cpu().numpy().view(np.uint32)
            assert np.array_equal(host, oracle.msm(s.cpu().numpy().view(np.uint32),
                                                   pts.cpu().numpy().view(np.uint32))), n
    assert not np.array_equal(results[0], results[1])
    ctx.close()


def test_noalloc_rejects_sizes_beyond_the_array():
    import torch
    from cusnarks_b200 import lib
    L = lib()
    n = L.cs_msm_g1_noalloc_max_terms() + 1
    # real buffers of the right size, so nothing could read out of bounds even if the
    # size check did not refuse the call
    s = torch.zeros((n, 8), dtype=torch.int32, device="cuda")
    p = torch.zeros((n, 16), dtype=torch.int32, device="cuda")
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = L.cs_msm_g1_noalloc(ctypes.c_void_p(s.data_ptr()), ctypes.c_void_p(p.data_ptr()), n,
                             ctypes.c_void_p(out.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == 2
    assert b"scratch" in L.cs_msm_g1_noalloc_error()
    assert not out.any()
