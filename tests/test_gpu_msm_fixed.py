"""Fixed-base (resident-table) multi-exponentiation: the table holds 2^(c j) P_i exactly,
and the MSM over the table equals the oracle's multi-exp of the original points, word for
word, for every window shape of the single-bucket-set reduction (1 to 4 levels)."""
import numpy as np
import pytest

from oracle.oracle import random_field, ints_to_limbs, limbs_to_int, R
from tests.gpu_common import random_points

pytestmark = pytest.mark.gpu

Q = 21888242871839275222246405745257275088696311157297823662689037894645226208583


@pytest.fixture(scope="module")
def ctx():
    from cusnarks_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def pts_g1(oracle):
    return random_points(oracle, np.random.Generator(np.random.PCG64(303)), 4096, ec2=False)


@pytest.fixture(scope="module")
def pts_g2(oracle):
    return random_points(oracle, np.random.Generator(np.random.PCG64(404)), 512, ec2=True)


def _inf(oracle, ec2=False):
    one = oracle.const(0)[0]
    if ec2:
        return np.concatenate([np.zeros(16, np.uint32), one, np.zeros(8, np.uint32)])
    return np.concatenate([np.zeros(8, np.uint32), one])


def fixed_msm(ctx, s, p, window, ec2=False, want_table=False):
    """Builds the table for points p and runs the fixed-base MSM with scalars s."""
    import torch
    n = s.shape[0]
    pw = 32 if ec2 else 16
    ds = torch.from_numpy(np.ascontiguousarray(s, dtype=np.uint32).view(np.int32)).cuda()
    dp = torch.from_numpy(np.ascontiguousarray(p, dtype=np.uint32).view(np.int32)).cuda()
    tab = torch.zeros(max(1, ctx.msm_fixed_table_points(n, window)) * pw, dtype=torch.int32, device="cuda")
    dout = torch.zeros(pw, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.msm_fixed_table_device(dp.data_ptr(), n, window, tab.data_ptr(), ec2)
    ctx.msm_fixed_device(ds.data_ptr(), tab.data_ptr(), n, window, dout.data_ptr(), ec2)
    ctx.sync()
    out = dout.cpu().numpy().view(np.uint32).copy()
    if want_table:
        return out, tab.cpu().numpy().view(np.uint32).reshape(-1, pw).copy()
    return out


@pytest.mark.parametrize("ec2,n,window", [(False, 64, 10), (True, 16, 8)])
def test_table_holds_window_multiples(ctx, oracle, pts_g1, pts_g2, ec2, n, window):
    p = (pts_g2 if ec2 else pts_g1)[:n].copy()
    p[5] = _inf(oracle, ec2)
    s = random_field(np.random.Generator(np.random.PCG64(1)), n, 1)
    _, tab = fixed_msm(ctx, s, p, window, ec2, want_table=True)
    W = ctx.msm_fixed_table_points(n, window) // n
    assert W == 254 // window + 1
    for j in range(W):
        k = np.tile(ints_to_limbs([pow(2, window * j, R)]), (n, 1))
        want = oracle.scmul(k, p, 1 if ec2 else 0)
        assert np.array_equal(tab[j * n:(j + 1) * n], want), j


@pytest.mark.parametrize("window", [6, 13, 16, 20, 22])
def test_fixed_g1_windows_match_oracle(ctx, oracle, pts_g1, window):
    """c = 6, 13: one reduction level; 16: two; 20: three; 22: four."""
    s = random_field(np.random.Generator(np.random.PCG64(window)), pts_g1.shape[0], 1)
    assert np.array_equal(fixed_msm(ctx, s, pts_g1, window), oracle.msm(s, pts_g1))


@pytest.mark.parametrize("n", [1, 3, 100, 1023])
def test_fixed_g1_ragged_auto_window(ctx, oracle, pts_g1, n):
    s = random_field(np.random.Generator(np.random.PCG64(n + 7)), n, 1)
    w = ctx.msm_fixed_window(n)
    assert 4 <= w <= 24
    assert np.array_equal(fixed_msm(ctx, s, pts_g1[:n], w), oracle.msm(s, pts_g1[:n]))


@pytest.mark.parametrize("window", [8, 0])
def test_fixed_g2_matches_oracle(ctx, oracle, pts_g2, window):
    n = pts_g2.shape[0]
    w = window or ctx.msm_fixed_window(n, True)
    s = random_field(np.random.Generator(np.random.PCG64(50 + window)), n, 1)
    assert np.array_equal(fixed_msm(ctx, s, pts_g2, w, ec2=True), oracle.msm(s, pts_g2, ec2=1))


def test_fixed_zero_scalars_infinity_duplicates(ctx, oracle, pts_g1):
    inf = _inf(oracle)
    assert np.array_equal(fixed_msm(ctx, np.zeros((64, 8), np.uint32), pts_g1[:64], 10), inf)
    P = pts_g1[7].copy()
    negP = P.copy()
    negP[8:] = ints_to_limbs([Q - limbs_to_int(P[8:])])[0]
    pts = np.stack([P] * 40 + [negP] * 40 + [inf] * 10 + list(pts_g1[100:110]))
    rng = np.random.Generator(np.random.PCG64(9))
    s = np.concatenate([np.tile(ints_to_limbs([12345]), (80, 1)), random_field(rng, 20, 1)])
    assert np.array_equal(fixed_msm(ctx, s, pts, 12), oracle.msm(s, pts))
    s2 = np.tile(ints_to_limbs([777]), (80, 1))
    assert np.array_equal(fixed_msm(ctx, s2, pts[:80], 12), inf)


def test_fixed_scalars_above_r_and_skewed(ctx, oracle, pts_g1):
    rng = np.random.Generator(np.random.PCG64(5))
    s = random_field(rng, 256, 1)
    big = []
    for i, row in enumerate(s):
        k, j = limbs_to_int(row), i % 6
        while k + j * R >= (1 << 256):
            j -= 1
        big.append(k + j * R)
    assert np.array_equal(fixed_msm(ctx, ints_to_limbs(big), pts_g1[:256], 11), oracle.msm(s, pts_g1[:256]))
    # all scalars equal: every window's digit of every term lands in the same few buckets
    se = np.tile(ints_to_limbs([0xdeadbeef12345]), (4096, 1))
    assert np.array_equal(fixed_msm(ctx, se, pts_g1, 20), oracle.msm(se, pts_g1))


def test_fixed_equals_generic_large(ctx):
    """2^17 terms, automatic windows: fixed-base and generic GPU MSMs agree."""
    import torch
    n = 1 << 17
    rng = np.random.Generator(np.random.PCG64(2024))
    s = random_field(rng, n, 1)
    k = random_field(rng, n, 1)
    # points k_i * G via the batched scalar multiplication kernel (one shared base)
    from tests.gpu_common import g1_generator_mont
    dk = torch.from_numpy(k.view(np.int32)).cuda()
    dg = torch.from_numpy(g1_generator_mont().view(np.int32)).cuda()
    dp = torch.zeros((n, 16), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.scmul_device(dk.data_ptr(), dg.data_ptr(), n, dp.data_ptr(), point_stride_words=0)
    ctx.sync()
    p = dp.cpu().numpy().view(np.uint32)
    gen = ctx.msm(s, p)
    w = ctx.msm_fixed_window(n)
    assert np.array_equal(fixed_msm(ctx, s, p, w), gen)


def _neg(p, ec2=False):
    """-P of an affine Montgomery point (y -> q - y per coordinate; 0 stays 0)."""
    out = p.copy()
    w = 16 if ec2 else 8
    for k in range(w // 8):
        y = limbs_to_int(p[w + 8 * k:w + 8 * (k + 1)])
        out[w + 8 * k:w + 8 * (k + 1)] = ints_to_limbs([(Q - y) % Q])[0]
    return out


@pytest.mark.parametrize("ec2,rounds", [(True, 1), (True, 2), (False, 1), (False, 2)])
def test_fixed_affine_rounds_match_oracle(ctx, oracle, pts_g1, pts_g2, ec2, rounds):
    """Batch-affine rounds forced on a fixed-base MSM: round one gathers table rows j*n + i
    through the sorted entries (k_affine_round with FIRST), later rounds their outputs.
    Many copies of P and -P under one scalar put equal points (doublings), opposite points
    (infinity inside the rounds) and their results side by side in the same buckets; points
    at infinity and zero scalars are among the terms."""
    pts = pts_g2 if ec2 else pts_g1
    inf = _inf(oracle, ec2)
    P = pts[3].copy()
    rest = list(pts[100:100 + 400])
    p = np.stack([P] * 48 + [_neg(P, ec2)] * 40 + [inf] * 8 + rest)
    rng = np.random.Generator(np.random.PCG64(700 + rounds + 10 * ec2))
    s = np.concatenate([np.tile(ints_to_limbs([0x1f2e3d4c5b6a79881726354]), (88, 1)),
                        random_field(rng, 8 + len(rest), 1)])
    s[100:104] = 0
    ctx.set_msm_affine_rounds(rounds)
    try:
        got = fixed_msm(ctx, s, p, 8, ec2)
        # everything cancels: equal numbers of P and -P under one scalar
        k = np.tile(ints_to_limbs([0xabcdef]), (80, 1))
        none = fixed_msm(ctx, k, np.stack([P] * 40 + [_neg(P, ec2)] * 40), 8, ec2)
    finally:
        ctx.set_msm_affine_rounds(-1)
    assert np.array_equal(got, oracle.msm(s, p, ec2=1 if ec2 else 0))
    assert np.array_equal(none, inf)
