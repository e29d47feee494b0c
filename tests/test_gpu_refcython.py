"""The reference's own Cython module, pycusnarks (src/cython/_cusnarks_kernel.pyx), built by
cusnarks_b200/refcython.py against this library, on the reference's golden vectors and on
fixtures the reference library produced: its wrappers ec_jacreduce_h (pyx:992), ntt_h /
intt_h (pyx:354 / :370), ntt_interpolandmul_h (pyx:479) and mpoly_eval_h (pyx:452) run
this library's GPU entry points and return the reference's answers word for word."""
import importlib
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pycusnarks():
    from cusnarks_b200 import refcython
    path = refcython.module_path()
    if path is None:
        pytest.skip("pycusnarks not built here: the reference tree was absent at build time")
    d = os.path.dirname(path)
    sys.path.insert(0, d)
    try:
        mod = importlib.import_module("pycusnarks")
    finally:
        sys.path.remove(d)
    return mod


def test_module_links_this_library(pycusnarks):
    maps = open("/proc/self/maps").read()
    ours = os.path.join("cusnarks_b200", "libcusnarks_b200.so")
    assert ours in maps
    assert "pycusnarks" in maps
    import subprocess
    need = subprocess.run(["ldd", pycusnarks.__file__], capture_output=True, text=True).stdout
    assert "libcusnarks_b200.so" in need and "libcusnarks.so" not in need


@pytest.mark.parametrize("ec2,name", [(0, "g1_msm_1024.npz"), (1, "g2_msm_1024.npz")])
def test_ec_jacreduce_h_golden(pycusnarks, golden, ec2, name):
    g = golden(name)
    scl = np.ascontiguousarray(g["scalars"].reshape(-1))
    pts = np.ascontiguousarray(g["points"].reshape(-1))
    # inscl, intbl, fname, offset, total_words, order, ec2, pidx, to_aff, add_in, strip_last, pippen
    out = pycusnarks.ec_jacreduce_h(scl, pts, b"", 0, 0, 6, ec2, 0, 1, 0, 1, 0)
    assert np.array_equal(np.asarray(out).reshape(-1), g["reduction"])


@pytest.mark.parametrize("L", [4, 7, 10])
def test_ntt_intt_h_reference_fixture(pycusnarks, oracle, golden, L):
    f = golden("ref_transforms.npz")
    roots = np.ascontiguousarray(oracle.find_roots(L))  # the wrapper takes L from the table
    A = np.ascontiguousarray(f[f"ntt_in_{L}"])
    fwd = pycusnarks.ntt_h(A.copy(), roots, 1, 1, 1, 1)
    assert np.array_equal(np.asarray(fwd).reshape(-1, 8), f[f"ntt_fwd_{L}"])
    for fmat, key in ((1, "ntt_inv_mont"), (0, "ntt_inv_ext")):
        inv = pycusnarks.intt_h(A.copy(), roots, 1, fmat, 1)
        assert np.array_equal(np.asarray(inv).reshape(-1, 8), f[f"{key}_{L}"]), fmat


@pytest.mark.parametrize("L", [4, 7, 10])
def test_ntt_interpolandmul_h_reference_fixture(pycusnarks, oracle, golden, L):
    from oracle.oracle import hstep_roots_table
    f = golden("ref_transforms.npz")
    table = np.ascontiguousarray(hstep_roots_table(oracle, L).reshape(-1))
    A = np.ascontiguousarray(f[f"hstep_A_{L}"].reshape(-1))
    B = np.ascontiguousarray(f[f"hstep_B_{L}"].reshape(-1))
    M = pycusnarks.ntt_interpolandmul_h(A, B, table, 2, 1)
    assert np.array_equal(np.asarray(M).reshape(-1, 8), f[f"hstep_M_{L}"])


@pytest.mark.parametrize("nv", [16, 300])
def test_mpoly_eval_h_reference_fixture(pycusnarks, golden, nv):
    f = golden("ref_transforms.npz")
    nc = int(f[f"mpoly_ncons_{nv}"][0])
    pin = np.ascontiguousarray(f[f"mpoly_pin_{nv}"])
    w = np.ascontiguousarray(f[f"mpoly_w_{nv}"])
    out = pycusnarks.mpoly_eval_h(w, pin, 0, nc, 0, nv, 1, 1)
    assert np.array_equal(np.asarray(out), f[f"mpoly_out_{nv}"])
