"""Point routines of the binding on the GPU against the reference library's outputs:
ec_jac2aff_h, ec_jacaddreduce_h, ec_jacscmul_h, ec_jacsc1mul_h, ec_isoncurve_h (G1 and G2).
Jacobian results are compared as points (the library returns them with Z = 1)."""
import numpy as np
import pytest

from cusnarks_b200 import lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ec2", [0, 1])
def test_point_routines_match_reference(golden, ec2):
    L = lib()
    g = golden("dropin.npz")
    pre = f"g{ec2 + 1}_"
    fw = 16 if ec2 else 8
    jac = np.ascontiguousarray(g[pre + "jac"])
    aff = np.ascontiguousarray(g[pre + "aff"])
    n = jac.shape[0]
    j2a = L.ec2_jac2aff_h if ec2 else L.ec_jac2aff_h
    red = L.ec2_jacaddreduce_h if ec2 else L.ec_jacaddreduce_h
    scm = L.ec2_jacscmul_h if ec2 else L.ec_jacscmul_h
    sc1 = L.ec2_jacsc1mul_h if ec2 else L.ec_jacsc1mul_h
    onc = L.ec2_isoncurve_h if ec2 else L.ec_isoncurve_h
    for strip in (0, 1):
        y = np.zeros((n, (2 if strip else 3) * fw), np.uint32)
        j2a(y.ctypes.data, jac.ctypes.data, n, 0, strip)
        assert L.cs_last_status() == 0
        assert np.array_equal(y, g[pre + f"jac2aff_{strip}"]), strip
    z = np.zeros(3 * fw, np.uint32)
    red(z.ctypes.data, jac.ctypes.data, n, 0, 1, 0, 1)
    assert np.array_equal(z[:2 * fw], g[pre + "reduce_jac"])
    z = np.zeros(3 * fw, np.uint32)
    red(z.ctypes.data, aff.ctypes.data, n, 0, 1, 1, 1)
    assert np.array_equal(z[:2 * fw], g[pre + "reduce_aff"])
    z = np.zeros((n, 3 * fw), np.uint32)
    scl = np.ascontiguousarray(g[pre + "scmul_scl"])
    scm(z.ctypes.data, scl.ctypes.data, jac.ctypes.data, n, 0, 0)
    assert np.array_equal(z[:, :2 * fw], g[pre + "scmul_aff"])
    x = np.concatenate([scl.reshape(-1), aff[0].reshape(-1)]).astype(np.uint32)
    z = np.zeros((n, 3 * fw), np.uint32)
    sc1(z.ctypes.data, x.ctypes.data, n, 0, 1)
    assert np.array_equal(z[:, :2 * fw], g[pre + "sc1mul_aff"])
    rows = list(aff) + [g[pre + "bad"]]
    flags = [int(onc(np.ascontiguousarray(r).ctypes.data, 1, 0)) for r in rows]
    flags += [int(onc(np.ascontiguousarray(r).ctypes.data, 0, 0)) for r in jac]
    assert flags == list(g[pre + "oncurve"])


@pytest.mark.parametrize("ec2", [0, 1])
def test_inittable_matches_reference(golden, ec2):
    """ec_inittable_h / ec2_inittable_h: subset-sum tables (affine and Jacobian rows, a
    partial last table), compared as points with the reference's (normalised by its own
    ec_jac2aff_h)."""
    L = lib()
    g = golden("dropin.npz")
    pre = f"g{ec2 + 1}_"
    fw = 16 if ec2 else 8
    fn = L.ec2_inittable_h if ec2 else L.ec_inittable_h
    for add_last, key, order in ((1, "aff", 3), (0, "jac", 4)):
        src = np.ascontiguousarray(g[pre + key][:10])
        ent = ((10 + order - 1) // order) << order
        tab = np.zeros((ent, 3 * fw), np.uint32)
        fn(src.ctypes.data, tab.ctypes.data, 10, order, 0, add_last)
        assert L.cs_last_status() == 0
        want = g[pre + f"inittable_{add_last}"]
        # Z = 1 rows are affine; the Jacobian infinity (0, 1, 0) is the affine infinity (0, 1)
        assert np.array_equal(tab[:, :2 * fw], want), add_last


@pytest.mark.parametrize("ec2", [0, 1])
def test_jacadd_jacdouble_match_reference(golden, ec2):
    L = lib()
    g = golden("dropin.npz")
    pre = f"g{ec2 + 1}_"
    fw = 16 if ec2 else 8
    jac = np.ascontiguousarray(g[pre + "jac"])
    n = jac.shape[0]
    add = L.ec2_jacadd_h if ec2 else L.ec_jacadd_h
    dbl = L.ec2_jacdouble_h if ec2 else L.ec_jacdouble_h
    for i in range(n):
        z = np.zeros(3 * fw, np.uint32)
        add(z.ctypes.data, np.ascontiguousarray(jac[i]).ctypes.data,
            np.ascontiguousarray(jac[(i + 1) % n]).ctypes.data, 0)
        assert np.array_equal(z[:2 * fw], g[pre + "jacadd"][i]), i
        z = np.zeros(3 * fw, np.uint32)
        dbl(z.ctypes.data, np.ascontiguousarray(jac[i]).ctypes.data, 0)
        assert np.array_equal(z[:2 * fw], g[pre + "jacdbl"][i]), i


def test_mpoly_montgomery_match_reference(golden):
    L = lib()
    g = golden("dropin.npz")
    p = np.ascontiguousarray(g["mpoly_in"]).copy()
    L.mpoly_to_montgomery_h(p.ctypes.data, 1)
    assert np.array_equal(p, g["mpoly_to"])
    L.mpoly_from_montgomery_h(p.ctypes.data, 1)
    assert np.array_equal(p, g["mpoly_from"])
