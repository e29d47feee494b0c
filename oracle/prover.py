"""CPU restatement of the reference's Groth16 proving sequence, and proof verification.

TEST INFRASTRUCTURE ONLY.  ``cpu_prove`` follows src/python/groth_prover.py pysnarkP_CPU
(:575-790: mpoly_eval of A and B, ntt_interpolandmul, the five multi-exponentiations with
the extension scalars [1, r], [1, s], [-rs]) and the final combination of gen_proof
(:1414-1453: pi_C = pi_C2 + pi_C + s pi_A + r pi_B1), calling the oracle's restatements of
the reference routines (cs_oracle.c).  ``verify`` checks the Groth16 pairing equation
with oracle/bn254.py.
"""
from __future__ import annotations

import numpy as np

from .oracle import Oracle, ints_to_limbs, limbs_to_int, from_mont_int, R
from . import bn254


def _ext(a: np.ndarray, rows) -> np.ndarray:
    return np.concatenate([np.asarray(a, dtype=np.uint32).reshape(-1, 8), ints_to_limbs(rows)])


def cpu_prove_stages(o: Oracle, pk: dict, w: np.ndarray, r: int, s: int, order: int = 6, ref=None,
                     threads: int = 0):
    """cpu_prove's sequence as separate stages [(name, fn)] sharing one state dict: running
    every fn once, in order, leaves the proof in state["proof"].  The stages are the
    reference's CPU steps (groth_prover.py:585-790): QAP evaluation of A and B, the H step,
    the A, B2 (G2), B1 and C multi-exponentiations, and the H multi-exponentiation with the
    final combination (:1414-1453).  The H step's roots table is made here, once, as the
    reference loads it once at start-up.  threads: host threads of the reference library's
    H step (0 = all)."""
    import os
    nv, npub, m = pk["n_vars"], pk["n_public"], pk["domain_size"]
    L = m.bit_length() - 1
    w = np.ascontiguousarray(w, dtype=np.uint32).reshape(-1, 8)
    eng = ref if ref is not None else o
    if ref is not None:
        from .oracle import hstep_roots_table
        roots = hstep_roots_table(o, L)
    else:
        roots = o.find_roots(L + 1)
    st = {}

    def qap():
        st["pA"] = eng.mpoly_eval(w[:nv], pk["polsA"], m, 0, nv, 1)
        st["pB"] = eng.mpoly_eval(w[:nv], pk["polsB"], m, 0, nv, 1)

    def hstep():
        if ref is not None:
            M = ref.interpolandmul(st["pA"], st["pB"], roots, L, 2, max_threads=threads or os.cpu_count() or 1)
        else:
            M = o.interpolandmul(st["pA"], st["pB"], roots, L, 2)
        st["polH"] = M[m:2 * m - 1]

    def msm_a():
        st["pi_a"] = eng.msm(_ext(w[:nv], [1, r]), pk["A"][:nv + 2], 0, order)

    def msm_b2():
        st["pi_b"] = eng.msm(_ext(w[:nv], [1, s]), pk["B2"][:nv + 2], 1, order)

    def msm_b1():
        st["pi_b1"] = eng.msm(_ext(w[:nv], [1, s]), pk["B1"][:nv + 2], 0, order)

    def msm_c():
        st["pi_c"] = eng.msm(w[npub + 1:nv], pk["C"][npub + 1:nv], 0, order)

    def msm_h_combine():
        neg_rs = (-(r * s)) % R
        hpts = np.concatenate([pk["hExps"][:m - 1].reshape(-1, 16), pk["delta_1"].reshape(-1, 16)])
        pi_c2 = eng.msm(_ext(st["polH"], [neg_rs]), hpts, 0, order)
        fin_s = ints_to_limbs([1, 1, s, r])
        fin_p = np.stack([pi_c2, st["pi_c"], st["pi_a"], st["pi_b1"]])
        pi_c = eng.msm(fin_s, fin_p, 0, 2)
        st["proof"] = np.concatenate([st["pi_a"], st["pi_b"], pi_c]).astype(np.uint32)

    stages = [("qap", qap), ("hstep", hstep), ("msm_A", msm_a), ("msm_B2", msm_b2), ("msm_B1", msm_b1),
              ("msm_C", msm_c), ("msm_H+combine", msm_h_combine)]
    return stages, st


def cpu_prove(o: Oracle, pk: dict, w: np.ndarray, r: int, s: int, order: int = 6, ref=None) -> np.ndarray:
    """pk: host arrays as cusnarks_b200.groth.pk_to_host returns them.  Returns 64 words:
    pi_A | pi_B | pi_C, affine Montgomery.  With ref (an oracle.RefLib), the QAP evaluation,
    H step and multi-exponentiations run in the reference's own library instead of the
    restatement (same sequence, same results)."""
    stages, st = cpu_prove_stages(o, pk, w, r, s, order, ref)
    for _, fn in stages:
        fn()
    return st["proof"]


def _g1(words):
    x, y = (from_mont_int(limbs_to_int(words[i * 8:(i + 1) * 8]), 0) for i in range(2))
    one = from_mont_int((1 << 256) % bn254.Q, 0)
    if x == 0 and y == 1:
        return None
    return (x, y)


def _g2(words):
    v = [from_mont_int(limbs_to_int(words[i * 8:(i + 1) * 8]), 0) for i in range(4)]
    if v[0] == 0 and v[1] == 0 and v[2] == 1 and v[3] == 0:
        return None
    return ((v[0], v[1]), (v[2], v[3]))


def verify(vk: dict, proof: np.ndarray, public_inputs) -> bool:
    """vk with affine Montgomery arrays (alpha_1, beta_2, gamma_2, delta_2, IC rows);
    proof = 64 words pi_A | pi_B | pi_C; public_inputs: normal-form limbs (n_public x 8)."""
    vkp = {"alpha_1": _g1(vk["alpha_1"]), "beta_2": _g2(vk["beta_2"]), "gamma_2": _g2(vk["gamma_2"]),
           "delta_2": _g2(vk["delta_2"]), "IC": [_g1(row) for row in np.asarray(vk["IC"]).reshape(-1, 16)]}
    pr = {"A": _g1(proof[:16]), "B": _g2(proof[16:48]), "C": _g1(proof[48:64])}
    pub = [1] + [limbs_to_int(row) for row in np.asarray(public_inputs).reshape(-1, 8)]
    return bn254.groth16_verify(vkp, pr, pub)
