"""Regenerate the golden fixtures under tests/golden/ from the reference tree.

Run in a container that has the reference mounted (default /root/reference) and the
reference CPU library built (``make -C oracle ref``):

    python tests/golden/make_golden.py [--ref DIR]  (default: $CUSNARKS_REF, else /root/reference)

Sources:
  * test/c/aux_data/test_scmul_samples.tbin, test_scmul_reduction_soln.tbin,
    test_scmul_soln.tbin (G1, 1024 points) and the test2_* G2 equivalents: raw uint32
    words (scalars, then affine Montgomery points; Jacobian per-point products).
  * test/c/test_utils_host.cpp, read as text: the field known answers A_test/B_test/C_test
    (Montgomery products mod r, :94-164), p_root128 and roots_128_test (:90, :165),
    ext_X_test / ext_X0X1_test (Fp2 products, :6395, :6700).
  * outputs of the reference CPU library itself (oracle/_ref) on small seeded inputs for
    ntt_h, intt_h, ntt_parallel_h, ntt_parallel2D_h, ntt_interpolandmul_server_h (with
    get_Mmul_h after it) and mpoly_eval_h.

The fixtures are what the GPU tests compare against on a machine without the reference.
"""
from __future__ import annotations

import argparse
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle.oracle import Oracle, RefLib, random_field, hstep_roots_table  # noqa: E402


def c_array(text: str, name: str) -> np.ndarray:
    i = text.index(f"static uint32_t {name}[]")
    body = text[text.index("{", i) + 1:text.index("};", i)]
    body = re.sub(r"//[^\n]*", "", body)
    vals = [int(v, 0) for v in re.findall(r"0x[0-9a-fA-F]+|\d+", body)]
    return np.array(vals, dtype=np.uint64).astype(np.uint32)


def make_mpoly(rng, nvars: int, ncons: int, nnz_per_var: int, oracle: Oracle):
    """Random mpoly in the reference layout (mpoly.cpp:195): [nVars][ncoeff_i..][per poly:
    constraint ids, then Montgomery values]."""
    words = [nvars]
    counts = rng.integers(0, nnz_per_var + 1, size=nvars)
    words += [int(c) for c in counts]
    body = []
    for i in range(nvars):
        c = int(counts[i])
        ids = rng.choice(ncons, size=c, replace=False) if c else np.zeros(0, np.int64)
        vals = oracle.to_mont(random_field(rng, c, 1), 1) if c else np.zeros((0, 8), np.uint32)
        body += [int(x) for x in ids]
        body += [int(x) for x in vals.reshape(-1)]
    return np.array(words + body, dtype=np.uint64).astype(np.uint32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("CUSNARKS_REF", "/root/reference"))
    args = ap.parse_args()
    aux = os.path.join(args.ref, "test", "c", "aux_data")
    src = open(os.path.join(args.ref, "test", "c", "test_utils_host.cpp")).read()
    oracle = Oracle()
    ref = RefLib.get()

    # ---- MSM golden files ---------------------------------------------------------
    n = 1024
    d = np.fromfile(os.path.join(aux, "test_scmul_samples.tbin"), dtype=np.uint32)
    red = np.fromfile(os.path.join(aux, "test_scmul_reduction_soln.tbin"), dtype=np.uint32)
    per = np.fromfile(os.path.join(aux, "test_scmul_soln.tbin"), dtype=np.uint32).reshape(n, 24)
    np.savez_compressed(os.path.join(HERE, "g1_msm_1024.npz"),
                        scalars=d[:n * 8].reshape(n, 8), points=d[n * 8:].reshape(n, 16),
                        reduction=red.reshape(16), per_point_jac=per[:64])
    d = np.fromfile(os.path.join(aux, "test2_scmul_samples.tbin"), dtype=np.uint32)
    red = np.fromfile(os.path.join(aux, "test2_scmul_reduction_soln.tbin"), dtype=np.uint32)
    per = np.fromfile(os.path.join(aux, "test2_scmul_soln.tbin"), dtype=np.uint32).reshape(n, 48)
    np.savez_compressed(os.path.join(HERE, "g2_msm_1024.npz"),
                        scalars=d[:n * 8].reshape(n, 8), points=d[n * 8:].reshape(n, 32),
                        reduction=red.reshape(32), per_point_jac=per[:64])

    # ---- field / roots known answers ----------------------------------------------
    np.savez_compressed(os.path.join(HERE, "field_kat.npz"),
                        A=c_array(src, "A_test").reshape(-1, 8),
                        B=c_array(src, "B_test").reshape(-1, 8),
                        C=c_array(src, "C_test").reshape(-1, 8),
                        p_root128=c_array(src, "p_root128").reshape(8),
                        roots_128=c_array(src, "roots_128_test").reshape(-1, 8),
                        ext_X=c_array(src, "ext_X_test").reshape(-1, 16),
                        ext_X0X1=c_array(src, "ext_X0X1_test").reshape(-1, 16))

    # ---- transforms computed by the reference library ------------------------------
    rng = np.random.Generator(np.random.PCG64(20240601))
    out = {}
    for L in (4, 7, 10):
        A = oracle.to_mont(random_field(rng, 1 << L, 1), 1)
        roots = oracle.find_roots(L + 1)       # table twice as long: exercises rstride = 2
        out[f"ntt_in_{L}"] = A
        out[f"ntt_fwd_{L}"] = ref.ntt(A, roots, L, 1, 2, 1, 1)
        out[f"ntt_inv_mont_{L}"] = ref.intt(A, roots, L, 2, 1, 1)
        out[f"ntt_inv_ext_{L}"] = ref.intt(A, roots, L, 2, 0, 1)
    for L in (4, 7, 10):
        A = oracle.to_mont(random_field(rng, 1 << L, 1), 1)
        B = oracle.to_mont(random_field(rng, 1 << L, 1), 1)
        table = hstep_roots_table(oracle, L)
        out[f"hstep_A_{L}"] = A
        out[f"hstep_B_{L}"] = B
        out[f"hstep_M_{L}"] = ref.interpolandmul(A, B, table, L, 2)
        out[f"hstep_Mmul_{L}"] = ref.mmul(L)
    for (nv, nc, k) in ((16, 16, 3), (300, 256, 4)):
        pin = make_mpoly(rng, nv, nc, k, oracle)
        w = random_field(rng, nv, 1)
        out[f"mpoly_pin_{nv}"] = pin
        out[f"mpoly_w_{nv}"] = w
        out[f"mpoly_out_{nv}"] = ref.mpoly_eval(w, pin, nc, 0, nv, 1)
        out[f"mpoly_ncons_{nv}"] = np.array([nc], np.uint32)
    # four-step transforms (ntt_parallel_h, ntt_parallel2D_h): (rows, cols, inner splits)
    for (nr, nc, fy, fx) in ((3, 4, 1, 2), (5, 5, 2, 3), (6, 4, 3, 2)):
        L = nr + nc
        A = oracle.to_mont(random_field(rng, 1 << L, 1), 1)
        roots = oracle.find_roots(L + 1)
        iroots = np.concatenate([roots[:1], roots[1:][::-1]])   # w^-j
        out[f"par_in_{nr}_{nc}"] = A
        for d in (1, -1):
            for mode in (0, 1):
                out[f"par_{nr}_{nc}_{d}_{mode}"] = ref.ntt_parallel(A, roots, nr, nc, 2, d, mode, 1)
        out[f"par2d_{nr}_{nc}_fwd"] = ref.ntt_parallel2D(A, roots, nr, fy, nc, fx, 2, 1, 1)
        out[f"par2d_{nr}_{nc}_inv"] = ref.ntt_parallel2D(A, iroots, nr, fy, nc, fx, 2, 1, 1)
        out[f"par2d_{nr}_{nc}_shape"] = np.array([nr, fy, nc, fx], np.uint32)
    np.savez_compressed(os.path.join(HERE, "ref_transforms.npz"), **out)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
