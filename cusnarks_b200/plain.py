"""Plain per-call GPU prover: the reference's proving flow, one drop-in call per step.

This is the reference's own sequence (src/python/groth_prover.py:575-790 pysnarkP_CPU and
the final combination :1414-1453 of gen_proof) driven through this library's drop-in entry
points, each a synchronous call on host memory, as the reference's Cython layer makes them:

    mpoly_eval_server_h            pA = A.w, pB = B.w               (QAP rows)
    ntt_interpolandmul_server_h    M = coefficients of A(x) B(x)    (roots table from host)
    ec_jacreduce_server_h  x 5     pi_A, pi_B (G2), pi_B1, pi_C, pi_C2; every call copies its
                                   scalars and proving-key points to the GPU, the key is not
                                   resident (the reference's GPU multi-exp does the same,
                                   groth_prover.py:1563 findECPointsDispatch)
    ec_jacreduce_server_h          pi_C = pi_C2 + pi_C + s pi_A + r pi_B1  (4-term multi-exp)

It is the comparison arm for the resident / served paths (cs_prove, cs_server_*): same
kernels underneath, no key residency, no fixed-base tables, no overlap.  Its proofs are
byte-identical to theirs.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import lib, JacaddReduced, MpolyEval, InterpolAndMul, CsError, CS_OK

R = 21888242871839275222246405745257275088548364400416034343698204186575808495617
MONT = 1 << 256


def _limbs(x: int) -> np.ndarray:
    return np.array([(x >> (32 * i)) & 0xffffffff for i in range(8)], dtype=np.uint32)


def _ext(a: np.ndarray, vals) -> np.ndarray:
    return np.concatenate([np.asarray(a, dtype=np.uint32).reshape(-1, 8), np.stack([_limbs(v) for v in vals])])


def roots_table(levels: int) -> np.ndarray:
    """The roots table the reference prover hands to ntt_interpolandmul for m = 2^levels
    (groth_prover.py:308-334): [2^(L+1) | 2^floor((L+1)/2) | 2^(...)] roots of unity
    (powers of 5^((r-1)/2^k), Montgomery), computed by the find_roots_h drop-in."""
    L = lib()
    nroots = levels + 1
    n2 = nroots // 2
    n3 = n2 + 1 if nroots % 2 else n2 - 1
    parts = []
    for k in (nroots, n2, n3):
        prim = _limbs(pow(5, (R - 1) >> k, R) * MONT % R)
        out = np.zeros((1 << k) * 8, dtype=np.uint32)
        L.find_roots_h(out.ctypes.data, prim.ctypes.data, 1 << k, 1)
        st = L.cs_ntt_last_status()
        if st != CS_OK:
            raise CsError(st, "find_roots_h failed")
        parts.append(out)
    return np.concatenate(parts)


class PlainProver:
    """pk: host arrays as groth.pk_to_host returns them."""

    def __init__(self, pk: dict):
        self.pk = pk
        self.m = pk["domain_size"]
        self.levels = self.m.bit_length() - 1
        self.roots = roots_table(self.levels)
        self.polsA = np.ascontiguousarray(pk["polsA"], dtype=np.uint32).reshape(-1)
        self.polsB = np.ascontiguousarray(pk["polsB"], dtype=np.uint32).reshape(-1)
        # the key's point arrays of the five multi-exponentiations, contiguous host arrays
        # made once per key (the reference loads its key once); each call still copies them
        # to the GPU, as the reference's multi-exp does
        nv, npub, m = pk["n_vars"], pk["n_public"], self.m
        key = lambda a, lo, hi, pw: np.ascontiguousarray(np.asarray(a, dtype=np.uint32).reshape(-1, pw)[lo:hi])  # noqa: E731
        self.pts_a = key(pk["A"], 0, nv + 2, 16)
        self.pts_b2 = key(pk["B2"], 0, nv + 2, 32)
        self.pts_b1 = key(pk["B1"], 0, nv + 2, 16)
        self.pts_c = key(pk["C"], npub + 1, nv, 16)
        self.pts_h = np.ascontiguousarray(np.concatenate([np.asarray(pk["hExps"], dtype=np.uint32).reshape(-1, 16)[:m - 1],
                                                          np.asarray(pk["delta_1"], dtype=np.uint32).reshape(-1, 16)]))

    def _mpoly(self, w, pin):
        nv = self.pk["n_vars"]
        out = np.zeros(self.m * 8, dtype=np.uint32)
        a = MpolyEval(out.ctypes.data, w.ctypes.data, pin.ctypes.data, 0, 0, nv, 0, 0, 1)
        lib().mpoly_eval_server_h(ctypes.byref(a))
        st = lib().cs_qap_last_status()
        if st != CS_OK:
            raise CsError(st, "mpoly_eval_server_h failed")
        return out

    def _msm(self, scl, pts, ec2=False):
        scl = np.ascontiguousarray(scl, dtype=np.uint32).reshape(-1)
        pts = np.ascontiguousarray(pts, dtype=np.uint32).reshape(-1)
        out = np.zeros(32 if ec2 else 16, dtype=np.uint32)
        a = JacaddReduced(out.ctypes.data, scl.ctypes.data, pts.ctypes.data, scl.size // 8, 1 if ec2 else 0,
                          0, None, 0, 0, 0, 0, 0, 0, 0, 0, 6, None)
        lib().ec_jacreduce_server_h(ctypes.byref(a))
        st = lib().cs_last_status()
        if st != CS_OK:
            raise CsError(st, lib().cs_last_error().decode() if lib().cs_last_error() else "msm failed")
        return out

    def prove(self, w, r: int, s: int) -> np.ndarray:
        """w: (n_vars, 8) normal form; r, s: ints.  Returns 64 words pi_A | pi_B | pi_C."""
        pk, m = self.pk, self.m
        nv, npub = pk["n_vars"], pk["n_public"]
        w = np.ascontiguousarray(w, dtype=np.uint32).reshape(-1, 8)[:nv]
        pA = self._mpoly(w, self.polsA)
        pB = self._mpoly(w, self.polsB)
        ncols = self.levels // 2
        a = InterpolAndMul(pA.ctypes.data, pB.ctypes.data, self.roots.ctypes.data, self.levels - ncols, ncols,
                           0, 0, self.levels, 2, 1, 0, 0, 0, 0)
        ptr = lib().ntt_interpolandmul_server_h(ctypes.byref(a))
        st = lib().cs_ntt_last_status()
        if st != CS_OK or not ptr:
            raise CsError(st, "ntt_interpolandmul_server_h failed")
        M = np.ctypeslib.as_array(ptr, shape=((2 * m) * 8,)).reshape(-1, 8)
        polH = M[m:2 * m - 1].copy()
        neg_rs = (-(r * s)) % R
        ws = _ext(w, [1, s])
        pi_a = self._msm(_ext(w, [1, r]), self.pts_a)
        pi_b = self._msm(ws, self.pts_b2, ec2=True)
        pi_b1 = self._msm(ws, self.pts_b1)
        pi_c = self._msm(w[npub + 1:nv], self.pts_c)
        pi_c2 = self._msm(_ext(polH, [neg_rs]), self.pts_h)
        fin = self._msm(np.stack([_limbs(1), _limbs(1), _limbs(s), _limbs(r)]),
                        np.stack([pi_c2, pi_c, pi_a, pi_b1]))
        return np.concatenate([pi_a, pi_b, fin]).astype(np.uint32)
