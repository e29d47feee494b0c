"""GPU field arithmetic (both multiplication variants) against the oracle, bit-exact."""
import ctypes

import numpy as np
import pytest

from oracle.oracle import random_field, ints_to_limbs, Q, R, MOD

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from cusnarks_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _edge(p):
    vals = [0, 1, 2, p - 1, p - 2, (1 << 256) % p, p >> 1, (p >> 1) + 1, 0xFFFFFFFF, 1 << 224]
    return ints_to_limbs(vals)


def _run(ctx, op, pidx, a, b=None, words=8):
    import torch
    da = torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b).view(np.int32)).cuda() if b is not None else None
    dout = torch.zeros_like(da)
    ctx.field_op_device(op, pidx, da.data_ptr(), db.data_ptr() if db is not None else 0,
                        dout.data_ptr(), a.shape[0])
    ctx.sync()
    return dout.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("pidx", [0, 1])
def test_binary_ops(ctx, oracle, pidx):
    rng = np.random.Generator(np.random.PCG64(31 + pidx))
    a = np.concatenate([random_field(rng, 4000, pidx), _edge(MOD[pidx])])
    b = np.concatenate([random_field(rng, 4000, pidx), _edge(MOD[pidx])[::-1]])
    want_mul = oracle.montmult(a, b, pidx)
    assert np.array_equal(_run(ctx, "mul", pidx, a, b), want_mul)
    assert np.array_equal(_run(ctx, "mul_dp52", pidx, a, b), want_mul)
    z_add = np.zeros_like(a); z_sub = np.zeros_like(a)
    P = ctypes.POINTER(ctypes.c_uint32)
    for i in range(a.shape[0]):
        oracle.lib.or_addm(z_add[i].ctypes.data_as(P), a[i].ctypes.data_as(P), b[i].ctypes.data_as(P), pidx)
        oracle.lib.or_subm(z_sub[i].ctypes.data_as(P), a[i].ctypes.data_as(P), b[i].ctypes.data_as(P), pidx)
    assert np.array_equal(_run(ctx, "add", pidx, a, b), z_add)
    assert np.array_equal(_run(ctx, "sub", pidx, a, b), z_sub)


@pytest.mark.parametrize("pidx", [0, 1])
def test_unary_ops(ctx, oracle, pidx):
    rng = np.random.Generator(np.random.PCG64(41 + pidx))
    a = np.concatenate([random_field(rng, 1000, pidx), _edge(MOD[pidx])])
    assert np.array_equal(_run(ctx, "sqr", pidx, a), oracle.montmult(a, a, pidx))
    assert np.array_equal(_run(ctx, "to_mont", pidx, a), oracle.to_mont(a, pidx))
    assert np.array_equal(_run(ctx, "from_mont", pidx, a), oracle.from_mont(a, pidx))
    inv = np.zeros_like(a)
    P = ctypes.POINTER(ctypes.c_uint32)
    for i in range(a.shape[0]):
        oracle.lib.or_montinv(inv[i].ctypes.data_as(P), a[i].ctypes.data_as(P), pidx)
    assert np.array_equal(_run(ctx, "inv", pidx, a), inv)


def test_field_known_answers(ctx, golden):
    kat = golden("field_kat.npz")
    # test_mul (reference test_utils_host.cpp:7160): montmult_h(A, B, MOD_FIELD) == C
    assert np.array_equal(_run(ctx, "mul", 1, kat["A"], kat["B"]), kat["C"])


def test_fq2_mul(ctx, oracle):
    rng = np.random.Generator(np.random.PCG64(51))
    a = random_field(rng, 2000, 0).reshape(-1, 16)
    b = random_field(rng, 2000, 0).reshape(-1, 16)
    want = np.zeros_like(a)
    P = ctypes.POINTER(ctypes.c_uint32)
    for i in range(a.shape[0]):
        oracle.lib.or_montmult_ext(want[i].ctypes.data_as(P), a[i].ctypes.data_as(P), b[i].ctypes.data_as(P), 0)
    assert np.array_equal(_run(ctx, "fq2_mul", 0, a, b), want)


def test_dropin_field_entry_points(oracle):
    from cusnarks_b200 import lib
    L = lib()
    rng = np.random.Generator(np.random.PCG64(61))
    a = random_field(rng, 64, 1); b = random_field(rng, 64, 1)
    out = np.zeros(8, np.uint32)
    L.montmult_h(out.ctypes.data, a[0].ctypes.data, b[0].ctypes.data, 1)
    assert L.cs_field_last_status() == 0
    assert np.array_equal(out, oracle.montmult(a[:1], b[:1], 1)[0])
    z = np.zeros_like(a)
    L.to_montgomeryN_h(z.ctypes.data, a.ctypes.data, 64, 1)
    assert np.array_equal(z, oracle.to_mont(a, 1))
    L.from_montgomeryN_h(z.ctypes.data, a.ctypes.data, 64, 1, 0)
    assert np.array_equal(z, oracle.from_mont(a, 1))
    L.from_montgomeryN_h(z.ctypes.data, a.ctypes.data, 64, 1, 2)
    assert L.cs_field_last_status() == 4  # unsupported option reported, no exit


@pytest.mark.parametrize("pidx", [0, 1])
def test_mul_dp52_lazy_inputs(ctx, oracle, pidx):
    """The radix-2^52 product takes lazily reduced operands in [0, 2p) (what the G1 bucket
    accumulation feeds it): x + p and y + p give the same canonical product as x and y."""
    rng = np.random.Generator(np.random.PCG64(51 + pidx))
    p = MOD[pidx]
    a = np.concatenate([random_field(rng, 2000, pidx), _edge(p)])
    b = np.concatenate([random_field(rng, 2000, pidx), _edge(p)[::-1]])
    want = oracle.montmult(a, b, pidx)

    def plus_p(x):
        vals = [int.from_bytes(r.tobytes(), "little") + p for r in x]
        return ints_to_limbs(vals)
    n = a.shape[0]
    mix = np.arange(n)
    a2 = np.where((mix & 1)[:, None] == 1, plus_p(a), a).astype(np.uint32)
    b2 = np.where((mix & 2)[:, None] == 2, plus_p(b), b).astype(np.uint32)
    assert np.array_equal(_run(ctx, "mul_dp52", pidx, a2, b2), want)


def _structured(p):
    """Operands in [0, 2p) at the edges of the radix-2^52 cut and of the lazy range: 0, 1,
    p - 1, p, p + 1, 2p - 1, 2p - 2, values at the 2^52, 2^104, 2^156, 2^208 limb boundaries
    (and those plus p), R mod p and its double."""
    vals = {0, 1, 2, p - 1, p, p + 1, 2 * p - 1, 2 * p - 2, (1 << 256) % p, (2 << 256) % p}
    for b in (52, 104, 156, 208):
        for v in ((1 << b) - 1, 1 << b, (1 << b) + 1, p - (1 << b), p + (1 << b), p + (1 << b) - 1):
            if 0 <= v < 2 * p:
                vals.add(v)
    return sorted(vals)


@pytest.mark.parametrize("pidx", [0, 1])
def test_mul_dp52_ten_million_products(ctx, oracle, pidx):
    """10^7 random products (half the operands lifted into [p, 2p)) plus every pair of the
    structured edge operands, radix-2^52 FP64-pipe product against the oracle's montmult_h
    restatement (ff.cpp:225), all words equal."""
    from oracle.oracle import _p
    p = MOD[pidx]
    n = 10_000_000
    rng = np.random.Generator(np.random.PCG64(1000 + pidx))
    a = random_field(rng, n, pidx)
    b = random_field(rng, n, pidx)
    # lift every other operand by p (a lazily reduced value, still below 2p < 2^256)
    pl = ints_to_limbs([p])[0].astype(np.uint64)
    for x, sel in ((a, slice(0, n, 2)), (b, slice(1, n, 3))):
        v = x[sel].astype(np.uint64)
        carry = np.zeros(v.shape[0], dtype=np.uint64)
        for i in range(8):
            t = v[:, i] + pl[i] + carry
            v[:, i] = t & 0xFFFFFFFF
            carry = t >> 32
        x[sel] = v.astype(np.uint32)
    e = ints_to_limbs(_structured(p))
    ea = np.repeat(e, e.shape[0], axis=0)
    eb = np.tile(e, (e.shape[0], 1))
    a = np.ascontiguousarray(np.concatenate([a, ea]))
    b = np.ascontiguousarray(np.concatenate([b, eb]))
    want = np.zeros_like(a)
    oracle.lib.or_montmult_batch(_p(want), _p(a), _p(b), ctypes.c_uint64(a.shape[0]), pidx)
    got = _run(ctx, "mul_dp52", pidx, a, b)
    bad = np.nonzero((got != want).any(axis=1))[0]
    assert bad.size == 0, (bad.size, bad[:5])
