"""GPU multi-exponentiation against the oracle and the reference golden vectors.

Bit-exact: results are affine Montgomery points and must match word for word.
"""
import numpy as np
import pytest

from oracle.oracle import random_field, ints_to_limbs, R, limbs_to_int
from tests.gpu_common import random_points

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from cusnarks_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def pts_g1(oracle):
    return random_points(oracle, np.random.Generator(np.random.PCG64(101)), 4096, ec2=False)


@pytest.fixture(scope="module")
def pts_g2(oracle):
    return random_points(oracle, np.random.Generator(np.random.PCG64(202)), 1024, ec2=True)


INF_G1 = None


@pytest.mark.parametrize("ec2,name", [(0, "g1_msm_1024.npz"), (1, "g2_msm_1024.npz")])
def test_msm_golden(ctx, golden, ec2, name):
    g = golden(name)
    out = ctx.msm(g["scalars"], g["points"], ec2=bool(ec2))
    assert np.array_equal(out, g["reduction"])


@pytest.mark.parametrize("ec2,name", [(0, "g1_msm_1024.npz"), (1, "g2_msm_1024.npz")])
def test_dropin_ec_jacreduce_h_golden(golden, ec2, name):
    from cusnarks_b200 import pycusnarks as pc
    g = golden(name)
    out = pc.ec_jacreduce_h(g["scalars"].reshape(-1), g["points"].reshape(-1), b"", 0, 0, 6,
                            ec2, 0, 1, 1, 1, 0)
    assert np.array_equal(out.reshape(-1), g["reduction"])


@pytest.mark.parametrize("window", [0, 4, 7, 10, 13, 16])
def test_msm_g1_random_windows(ctx, oracle, pts_g1, window):
    rng = np.random.Generator(np.random.PCG64(window + 1))
    s = random_field(rng, pts_g1.shape[0], 1)
    assert np.array_equal(ctx.msm(s, pts_g1, window=window), oracle.msm(s, pts_g1))


@pytest.mark.parametrize("n", [1, 2, 3, 31, 100, 1023])
def test_msm_g1_ragged_sizes(ctx, oracle, pts_g1, n):
    rng = np.random.Generator(np.random.PCG64(n))
    s = random_field(rng, n, 1)
    assert np.array_equal(ctx.msm(s, pts_g1[:n]), oracle.msm(s, pts_g1[:n]))


@pytest.mark.parametrize("window", [0, 5, 11])
def test_msm_g2_random(ctx, oracle, pts_g2, window):
    rng = np.random.Generator(np.random.PCG64(77 + window))
    s = random_field(rng, pts_g2.shape[0], 1)
    assert np.array_equal(ctx.msm(s, pts_g2, ec2=True, window=window), oracle.msm(s, pts_g2, ec2=1))


def test_msm_empty_and_zero(ctx, oracle, pts_g1):
    one = oracle.const(0)[0]
    inf = np.concatenate([np.zeros(8, np.uint32), one])
    assert np.array_equal(ctx.msm(np.zeros((0, 8), np.uint32), np.zeros((0, 16), np.uint32)), inf)
    z = np.zeros((64, 8), np.uint32)
    assert np.array_equal(ctx.msm(z, pts_g1[:64]), inf)


def test_msm_scalars_above_r(ctx, oracle, pts_g1):
    """Scalars are full 256-bit values (the golden file has some); k and k + j*r agree."""
    rng = np.random.Generator(np.random.PCG64(5))
    s = random_field(rng, 256, 1)
    big = []
    for i, row in enumerate(s):
        k = limbs_to_int(row)
        j = i % 6
        while k + j * R >= (1 << 256):
            j -= 1
        big.append(k + j * R)
    sb = ints_to_limbs(big)
    ref = oracle.msm(s, pts_g1[:256])
    assert np.array_equal(ctx.msm(sb, pts_g1[:256]), ref)
    assert np.array_equal(oracle.msm(sb, pts_g1[:256]), ref)


def test_msm_duplicates_cancellation_and_infinity(ctx, oracle, pts_g1):
    """Same point many times (bucket doublings), P and -P (cancellation), infinity points."""
    one = oracle.const(0)[0]
    inf = np.concatenate([np.zeros(8, np.uint32), one])
    P = pts_g1[7].copy()
    negP = P.copy()
    q = 21888242871839275222246405745257275088696311157297823662689037894645226208583
    negP[8:] = ints_to_limbs([q - limbs_to_int(P[8:])])[0]
    pts = np.stack([P] * 40 + [negP] * 40 + [inf] * 10 + list(pts_g1[100:110]))
    rng = np.random.Generator(np.random.PCG64(9))
    s = np.concatenate([np.tile(ints_to_limbs([12345]), (40, 1)), np.tile(ints_to_limbs([12345]), (40, 1)),
                        random_field(rng, 10, 1), random_field(rng, 10, 1)])
    assert np.array_equal(ctx.msm(s, pts), oracle.msm(s, pts))
    # pure cancellation -> infinity
    s2 = np.tile(ints_to_limbs([777]), (80, 1))
    assert np.array_equal(ctx.msm(s2, pts[:80]), inf)


def _glv_lambda():
    """lambda of the G1 endomorphism (phi(P) = lambda P), from the split's lattice vector
    (a1, b1): a1 + b1 lambda = 0 mod r."""
    a1 = 0x89d3256894d213e3
    b1 = -0x6f4d8248eeb859fc8211bbeb7d4f1128
    lam = (-a1 * pow(b1, -1, R)) % R
    assert (lam * lam + lam + 1) % R == 0
    return lam


def test_msm_glv_edge_scalars(ctx, oracle, pts_g1):
    """G1 MSMs split every scalar as k1 + k2 lambda: scalars whose halves are zero, one,
    negative or at the 2^127 bound, each alone (one term) and all together."""
    lam = _glv_lambda()
    ks = [1, 2, R - 1, R - 2, lam, lam + 1, lam - 1, R - lam, (lam * lam) % R, 2 * lam % R,
          (1 << 127) - 1, 1 << 127, (1 << 128) - 1, 1 << 200, (1 << 253) + 12345, R + 5,
          (1 << 256) - 1, 0x0be4e1541221250b6f4d8248eeb859fd, (R - 1) // 2, (R + 1) // 2]
    s = ints_to_limbs(ks)
    P = pts_g1[:len(ks)]
    for i in range(len(ks)):
        assert np.array_equal(ctx.msm(s[i:i + 1], P[i:i + 1]), oracle.msm(s[i:i + 1], P[i:i + 1])), hex(ks[i])
    assert np.array_equal(ctx.msm(s, P), oracle.msm(s, P))
    for w in (5, 11, 16):
        assert np.array_equal(ctx.msm(s, P, window=w), oracle.msm(s, P)), w


def test_msm_skewed_scalars_one_bucket(ctx, oracle, pts_g1):
    """All scalars equal: every entry lands in one bucket per window (split tasks)."""
    s = np.tile(ints_to_limbs([0xdeadbeef12345]), (4096, 1))
    assert np.array_equal(ctx.msm(s, pts_g1, window=12), oracle.msm(s, pts_g1))
    s1 = np.tile(ints_to_limbs([1]), (4096, 1))
    assert np.array_equal(ctx.msm(s1, pts_g1), oracle.msm(s1, pts_g1))


def test_msm_device_pointers_torch(ctx, oracle, pts_g1):
    import torch
    rng = np.random.Generator(np.random.PCG64(55))
    s = random_field(rng, 2048, 1)
    ds = torch.from_numpy(s.view(np.int32)).cuda()
    dp = torch.from_numpy(np.ascontiguousarray(pts_g1[:2048]).view(np.int32)).cuda()
    dout = torch.zeros(16, dtype=torch.int32, device="cuda")
    ctx.msm_device(ds.data_ptr(), dp.data_ptr(), 2048, dout.data_ptr())
    ctx.sync()
    got = dout.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, oracle.msm(s, pts_g1[:2048]))


@pytest.mark.parametrize("ec2", [0, 1])
def test_scmul_matches_oracle(ctx, oracle, golden, ec2):
    """Batched k_i * P_i (golden scalars include full 256-bit values) and fixed base."""
    import torch
    g = golden("g2_msm_1024.npz" if ec2 else "g1_msm_1024.npz")
    n = 256
    s = np.ascontiguousarray(g["scalars"][:n])
    p = np.ascontiguousarray(g["points"][:n])
    pw = p.shape[1]
    ds = torch.from_numpy(s.view(np.int32)).cuda()
    dp = torch.from_numpy(p.view(np.int32)).cuda()
    dout = torch.zeros((n, pw), dtype=torch.int32, device="cuda")
    ctx.scmul_device(ds.data_ptr(), dp.data_ptr(), n, dout.data_ptr(), ec2=bool(ec2))
    ctx.sync()
    assert np.array_equal(dout.cpu().numpy().view(np.uint32), oracle.scmul(s, p, ec2))
    # fixed base: every scalar times point 3
    dout.zero_()
    ctx.scmul_device(ds.data_ptr(), dp[3].data_ptr(), n, dout.data_ptr(), ec2=bool(ec2),
                     point_stride_words=0)
    ctx.sync()
    assert np.array_equal(dout.cpu().numpy().view(np.uint32), oracle.scmul(s, p[3:4], ec2))


@pytest.mark.parametrize("rounds", [0, 1, 3, 6])
def test_msm_affine_rounds(ctx, oracle, pts_g1, pts_g2, rounds):
    """Batch-affine halving rounds before the XYZZ accumulation: same results for any number
    of rounds, including equal points (doubling), P + (-P) (infinity inside a round), zero
    scalars, one giant bucket (all scalars equal) and G2."""
    one = oracle.const(0)[0]
    inf = np.concatenate([np.zeros(8, np.uint32), one])
    q = 21888242871839275222246405745257275088696311157297823662689037894645226208583
    ctx.set_msm_affine_rounds(rounds)
    try:
        rng = np.random.Generator(np.random.PCG64(700 + rounds))
        s = random_field(rng, pts_g1.shape[0], 1)
        assert np.array_equal(ctx.msm(s, pts_g1, window=8), oracle.msm(s, pts_g1))
        P = pts_g1[7].copy()
        negP = P.copy()
        negP[8:] = ints_to_limbs([q - limbs_to_int(P[8:])])[0]
        pts = np.stack([P] * 64 + [negP] * 63 + [inf] * 5 + list(pts_g1[100:164]))
        sc = np.concatenate([np.tile(ints_to_limbs([424242]), (127, 1)), random_field(rng, 5, 1),
                             random_field(rng, 64, 1)])
        sc[130] = 0
        assert np.array_equal(ctx.msm(sc, pts, window=6), oracle.msm(sc, pts))
        s1 = np.tile(ints_to_limbs([0xdeadbeef12345]), (4096, 1))
        assert np.array_equal(ctx.msm(s1, pts_g1, window=10), oracle.msm(s1, pts_g1))
        s2 = random_field(rng, pts_g2.shape[0], 1)
        assert np.array_equal(ctx.msm(s2, pts_g2, ec2=True, window=6), oracle.msm(s2, pts_g2, ec2=1))
    finally:
        ctx.set_msm_affine_rounds(-1)
