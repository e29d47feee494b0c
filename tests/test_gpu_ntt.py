"""GPU NTT / INTT / H step against the reference fixtures and the oracle (bit-exact)."""
import ctypes

import numpy as np
import pytest

from oracle.oracle import random_field, hstep_roots_table

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from cusnarks_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _lib():
    from cusnarks_b200 import lib
    return lib()


@pytest.mark.parametrize("L", [4, 7, 10])
def test_dropin_ntt_intt_reference_fixture(oracle, golden, L):
    """ntt_h / intt_h through the C ABI reproduce the reference library's outputs."""
    f = golden("ref_transforms.npz")
    L_ = _lib()
    roots = np.ascontiguousarray(oracle.find_roots(L + 1))
    A = np.ascontiguousarray(f[f"ntt_in_{L}"])
    a = A.copy()
    L_.ntt_h(a.ctypes.data, roots.ctypes.data, L, 1, 2, 1, 1)
    assert L_.cs_ntt_last_status() == 0
    assert np.array_equal(a, f[f"ntt_fwd_{L}"])
    for fmat, key in ((1, "ntt_inv_mont"), (0, "ntt_inv_ext")):
        a = A.copy()
        L_.intt_h(a.ctypes.data, roots.ctypes.data, fmat, L, 2, 1)
        assert np.array_equal(a, f[f"{key}_{L}"])


@pytest.mark.parametrize("L,astride,rstride", [(1, 1, 1), (2, 1, 4), (11, 1, 1), (12, 2, 1), (15, 1, 2), (21, 1, 1)])
def test_dropin_ntt_sizes_against_oracle(oracle, L, astride, rstride):
    rng = np.random.Generator(np.random.PCG64(100 + L))
    n = 1 << L
    roots = np.ascontiguousarray(oracle.find_roots(L + (rstride.bit_length() - 1)))
    A = oracle.to_mont(random_field(rng, n * astride, 1), 1)
    L_ = _lib()
    for direction in (1, -1):
        a = A.copy()
        L_.ntt_h(a.ctypes.data, roots.ctypes.data, L, astride, rstride, direction, 1)
        assert L_.cs_ntt_last_status() == 0
        want = oracle.ntt(A, roots, L, astride, rstride, direction, 1)
        assert np.array_equal(a, want), (L, direction)


def test_find_roots(oracle, golden):
    kat = golden("field_kat.npz")
    L_ = _lib()
    out = np.zeros((128, 8), np.uint32)
    p = np.ascontiguousarray(kat["p_root128"])
    L_.find_roots_h(out.ctypes.data, p.ctypes.data, 128, 1)
    assert np.array_equal(out, kat["roots_128"])


@pytest.mark.parametrize("L", [4, 7, 10])
def test_dropin_interpolandmul_reference_fixture(oracle, golden, L):
    from cusnarks_b200._lib import InterpolAndMul
    f = golden("ref_transforms.npz")
    L_ = _lib()
    table = np.ascontiguousarray(hstep_roots_table(oracle, L))
    A = np.ascontiguousarray(f[f"hstep_A_{L}"]); B = np.ascontiguousarray(f[f"hstep_B_{L}"])
    args = InterpolAndMul(A.ctypes.data, B.ctypes.data, table.ctypes.data, L - L // 2, L // 2, 0, 0, L, 2, 1, 8, 0, 0, 0)
    ptr = L_.ntt_interpolandmul_server_h(ctypes.byref(args))
    assert ptr and L_.cs_ntt_last_status() == 0
    M = np.ctypeslib.as_array(ptr, shape=((2 << L) * 8,)).copy().reshape(-1, 8)
    assert np.array_equal(M, f[f"hstep_M_{L}"])
    assert np.array_equal(A, f[f"hstep_A_{L}"])  # inputs untouched


@pytest.mark.parametrize("nr,nc", [(3, 4), (5, 5), (6, 4)])
def test_dropin_ntt_parallel_reference_fixture(oracle, golden, nr, nc):
    """ntt_parallel_h (both fft modes and directions) and ntt_parallel2D_h (forward table and
    inverse table, direction 1) reproduce the reference library's four-step outputs."""
    f = golden("ref_transforms.npz")
    L_ = _lib()
    L = nr + nc
    roots = np.ascontiguousarray(oracle.find_roots(L + 1))
    iroots = np.ascontiguousarray(np.concatenate([roots[:1], roots[1:][::-1]]))
    A = np.ascontiguousarray(f[f"par_in_{nr}_{nc}"])
    for d in (1, -1):
        for mode in (0, 1):
            a = A.copy()
            L_.ntt_parallel_h(a.ctypes.data, roots.ctypes.data, nr, nc, 2, d, mode, 1)
            assert L_.cs_ntt_last_status() == 0
            assert np.array_equal(a, f[f"par_{nr}_{nc}_{d}_{mode}"]), (d, mode)
    _, fy, _, fx = (int(x) for x in f[f"par2d_{nr}_{nc}_shape"])
    for tab, key in ((roots, "fwd"), (iroots, "inv")):
        a = A.copy()
        L_.ntt_parallel2D_h(a.ctypes.data, tab.ctypes.data, nr, fy, nc, fx, 2, 1, 1)
        assert L_.cs_ntt_last_status() == 0
        assert np.array_equal(a, f[f"par2d_{nr}_{nc}_{key}"]), key
    a = A.copy()
    L_.ntt_parallel2D_h(a.ctypes.data, roots.ctypes.data, nr, fy, nc, fx, 2, -1, 1)
    assert L_.cs_ntt_last_status() != 0 and np.array_equal(a, A)  # not a transform in the reference


@pytest.mark.parametrize("L", [4, 7, 10])
def test_dropin_get_mmul_reference_fixture(oracle, golden, L):
    """get_Mmul_h after an H step: the reference's pre-transpose matrix of the result."""
    from cusnarks_b200._lib import InterpolAndMul
    f = golden("ref_transforms.npz")
    L_ = _lib()
    table = np.ascontiguousarray(hstep_roots_table(oracle, L))
    A = np.ascontiguousarray(f[f"hstep_A_{L}"]); B = np.ascontiguousarray(f[f"hstep_B_{L}"])
    args = InterpolAndMul(A.ctypes.data, B.ctypes.data, table.ctypes.data, L - L // 2, L // 2, 0, 0, L, 2, 1, 8, 0, 0, 0)
    assert L_.ntt_interpolandmul_server_h(ctypes.byref(args))
    ptr = L_.get_Mmul_h()
    assert ptr
    M = np.ctypeslib.as_array(ptr, shape=((2 << L) * 8,)).copy().reshape(-1, 8)
    assert np.array_equal(M, f[f"hstep_Mmul_{L}"])


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


@pytest.mark.parametrize("L", [3, 11, 16, 20])
def test_native_ntt_roundtrip_and_oracle(ctx, oracle, L):
    import torch
    rng = np.random.Generator(np.random.PCG64(7 + L))
    n = 1 << L
    A = oracle.to_mont(random_field(rng, n, 1), 1)
    dA = _dev(A)
    dF = torch.empty_like(dA)
    ctx.ntt_device(dA.data_ptr(), dF.data_ptr(), L, 1)
    dB = torch.empty_like(dA)
    ctx.ntt_device(dF.data_ptr(), dB.data_ptr(), L, -1, fmat=1)
    ctx.sync()
    assert np.array_equal(dB.cpu().numpy().view(np.uint32), A)  # round trip
    if L <= 16:
        roots = oracle.find_roots(L)
        assert np.array_equal(dF.cpu().numpy().view(np.uint32), oracle.ntt(A, roots, L, 1, 1, 1, 1))


@pytest.mark.parametrize("L", [5, 12])
def test_native_hstep_variants(ctx, oracle, L):
    import torch
    rng = np.random.Generator(np.random.PCG64(17 + L))
    m = 1 << L
    A = oracle.to_mont(random_field(rng, m, 1), 1)
    B = oracle.to_mont(random_field(rng, m, 1), 1)
    C = oracle.to_mont(random_field(rng, m, 1), 1)
    dA, dB, dC = _dev(A), _dev(B), _dev(C)
    dM = torch.zeros((2 * m, 8), dtype=torch.int32, device="cuda")
    dH = torch.zeros((m, 8), dtype=torch.int32, device="cuda")
    ctx.hstep_device(0, dA.data_ptr(), dB.data_ptr(), 0, L, dM.data_ptr())
    ctx.hstep_device(1, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), L, dH.data_ptr())
    ctx.sync()
    roots = oracle.find_roots(L + 1)
    assert np.array_equal(dM.cpu().numpy().view(np.uint32), oracle.interpolandmul(A, B, roots, L, 2))
    assert np.array_equal(dH.cpu().numpy().view(np.uint32), oracle.hstep_coset(A, B, C, L))
    # satisfying input: both variants give the same quotient
    C2 = oracle.montmult(A, B, 1)
    dC2 = _dev(C2)
    ctx.hstep_device(1, dA.data_ptr(), dB.data_ptr(), dC2.data_ptr(), L, dH.data_ptr())
    ctx.sync()
    H = dH.cpu().numpy().view(np.uint32)
    M = dM.cpu().numpy().view(np.uint32)
    assert np.array_equal(H[:m - 1], M[m:2 * m - 1]) and not H[m - 1].any()
