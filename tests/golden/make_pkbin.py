"""Regenerate tests/golden/pk_files.npz: a proving key written by the reference's own writer
and a witness file written by the reference's own C routine.

    python tests/golden/make_pkbin.py [--ref DIR]  (default: $CUSNARKS_REF, else /root/reference)

* Proving key: src/python/pysnarks_utils.py pkvars_to_bin(FMT_MONT, EC_T_AFFINE, pk, ext=True)
  imported from the reference tree.  The module imports Python-2 compatibility packages
  (past, future) that are not installed here; they are replaced by minimal shims (range,
  int, str) that the writer's numpy code never reaches.  Inputs: a small seeded key (nVars 20,
  nPublic 1, domain 32) whose points are multiples of the generators computed by the oracle
  and whose mpolys have random Montgomery coefficients.
* Witness: writeWitnessFile_h (src/cuda/file_utils.cpp:583) from the reference CPU library
  (oracle/_ref, `make -C oracle ref`).
"""
from __future__ import annotations

import argparse
import ctypes
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle.oracle import Oracle, RefLib, random_field, G1_GEN, G2_GEN, ints_to_limbs, to_mont_int  # noqa: E402
from cusnarks_b200.groth import mpoly_from_entries  # noqa: E402  (pure numpy)


def _shim_py2_compat():
    pb = types.ModuleType("past.builtins")
    pb.xrange, pb.long, pb.basestring, pb.unicode = range, int, str, str
    p = types.ModuleType("past")
    p.builtins = pb
    sys.modules.setdefault("past", p)
    sys.modules.setdefault("past.builtins", pb)

    class Stub(types.ModuleType):
        def __getattr__(self, name):
            if name.startswith("__"):
                raise AttributeError(name)
            return lambda *a, **k: None
    for name in ("future", "future.builtins", "future.builtins.misc"):
        sys.modules.setdefault(name, Stub(name))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("CUSNARKS_REF", "/root/reference"))
    args = ap.parse_args()
    o = Oracle()
    rng = np.random.Generator(np.random.PCG64(2025))
    nv, npub, bits = 20, 1, 5
    m = 1 << bits
    g1 = np.concatenate([ints_to_limbs([to_mont_int(c, 0)]) for c in G1_GEN]).reshape(1, 16)
    g2 = np.concatenate([ints_to_limbs([to_mont_int(c, 0) for c in xy]) for xy in G2_GEN]).reshape(1, 32)

    def g1pts(n):
        return o.scmul(random_field(rng, n, 1), g1, 0).reshape(-1, 16)

    def g2pts(n):
        return o.scmul(random_field(rng, n, 1), g2, 1).reshape(-1, 32)

    A, B1, C, H = g1pts(nv), g1pts(nv), g1pts(nv), g1pts(m + 1)
    B2 = g2pts(nv)
    alfa_1, beta_1, delta_1 = g1pts(1), g1pts(1), g1pts(1)
    beta_2, delta_2 = g2pts(1), g2pts(1)
    ents = 3 * (m - npub - 1)
    cons = np.repeat(np.arange(m - npub - 1, dtype=np.uint32), 3)
    polsA = mpoly_from_entries(nv, rng.integers(0, nv, ents).astype(np.uint32), cons,
                               o.to_mont(random_field(rng, ents, 1), 1))
    polsB = mpoly_from_entries(nv, rng.integers(0, nv, ents).astype(np.uint32), cons,
                               o.to_mont(random_field(rng, ents, 1), 1))
    R = 21888242871839275222246405745257275088548364400416034343698204186575808495617
    Q = 21888242871839275222246405745257275088696311157297823662689037894645226208583

    _shim_py2_compat()
    sys.path.insert(0, os.path.join(args.ref, "src", "python"))
    import pysnarks_utils as pu  # noqa: E402
    rows = lambda a: np.ascontiguousarray(a, dtype=np.uint32).reshape(-1, 8)  # noqa: E731
    pk = {
        "nWords": 0, "Rbitlen": 256, "k_ecformat": 2, "nVars": nv, "nPublic": npub, "domainBits": bits,
        "domainSize": m, "field_r": ints_to_limbs([R])[0], "group_q": ints_to_limbs([Q])[0],
        "polsA": polsA, "polsB": polsB, "polsA_nWords": polsA.size, "polsB_nWords": polsB.size,
        "alfa_1": rows(alfa_1), "beta_1": rows(beta_1), "delta_1": rows(delta_1),
        "beta_2": rows(beta_2), "delta_2": rows(delta_2),
        "A": rows(A), "B1": rows(B1), "B2": rows(B2), "C": rows(C), "hExps": rows(H),
        "A_nWords": A.size, "B1_nWords": B1.size, "B2_nWords": B2.size, "C_nWords": C.size,
        "hExps_nWords": H.size,
    }
    pk_bin = np.asarray(pu.pkvars_to_bin(1, 2, dict(pk), ext=True), dtype=np.uint32)

    # witness through the reference C routine
    w = random_field(rng, nv, 1)
    ref = RefLib.get()
    fn = ref.lib._Z18writeWitnessFile_hPjPKcy
    fn.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_ulonglong]
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "w.bin")
        wc = np.ascontiguousarray(w)
        fn(wc.ctypes.data, path.encode(), nv)
        ctypes.CDLL(None).fflush(None)  # the routine leaves its FILE open: flush it
        wit_bin = np.fromfile(path, dtype="<u4")
    np.savez_compressed(os.path.join(HERE, "pk_files.npz"), pk_bin=pk_bin, n_vars=nv, n_public=npub, domain=m,
                        A=A, B1=B1, B2=B2, C=C, hExps=H, alfa_1=alfa_1, beta_1=beta_1, delta_1=delta_1,
                        beta_2=beta_2, delta_2=delta_2, polsA=polsA, polsB=polsB, witness=w, witness_bin=wit_bin)
    print("pk words", pk_bin.size, "witness words", wit_bin.size)


if __name__ == "__main__":
    main()
