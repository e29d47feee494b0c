"""The CPU prover restatement and the pairing check, on a small circuit built on the CPU.

CPU only: a tiny R1CS and its Groth16 key are built with Python integers and the oracle's
fixed-base multiplication; the restated proving sequence must produce a proof that passes
the BN254 pairing check, that fails for a wrong public input, and that is identical when
the reference's own library (oracle/_ref) computes the QAP evaluation, H step and
multi-exponentiations.
"""
import numpy as np
import pytest

from oracle.oracle import ints_to_limbs, limbs_to_int, R, to_mont_int, RefLib
from oracle.prover import cpu_prove, verify
from cusnarks_b200.groth import mpoly_from_entries
from tests.gpu_common import g1_generator_mont, g2_generator_mont


def _tiny_groth(o, L=4, seed=5, npub=1, nin=4):
    rng = np.random.default_rng(seed)
    m = 1 << L
    nc = m - npub - 1
    nv = nin + nc
    rnd = lambda: int(rng.integers(1, 1 << 62)) * 998244353 % R  # noqa: E731
    w = [1] + [rnd() for _ in range(nin - 1)] + [0] * nc
    arows, brows = [], []
    for c in range(nc):
        hi = nin + c
        a = [(int(rng.integers(0, hi)), rnd()) for _ in range(3)]
        b = [(int(rng.integers(0, hi)), rnd()) for _ in range(3)]
        arows.append(a)
        brows.append(b)
        w[nin + c] = (sum(cf * w[i] for i, cf in a) % R) * (sum(cf * w[i] for i, cf in b) % R) % R

    def ent(rows, extra=()):
        W, C, V = [], [], []
        for c, row in enumerate(rows):
            for i, cf in row:
                W.append(i); C.append(c); V.append(to_mont_int(cf, 1))
        for i, c, cf in extra:
            W.append(i); C.append(c); V.append(to_mont_int(cf, 1))
        return np.array(W, np.int64), np.array(C, np.uint32), ints_to_limbs(V)

    polsA = mpoly_from_entries(nv, *ent(arows, [(i, nc + i, 1) for i in range(npub + 1)]))
    polsB = mpoly_from_entries(nv, *ent(brows))
    t, al, be, ga, de = [rnd() for _ in range(5)]
    from oracle.oracle import from_mont_int
    omega = from_mont_int(limbs_to_int(o.find_roots(L)[1]), 1)
    Lc = [pow(omega, c, R) * (pow(t, m, R) - 1) * pow(m * (t - pow(omega, c, R)), -1, R) % R for c in range(m)]

    def wire_eval(entries):
        out = [0] * nv
        for i, c, cf in entries:
            out[i] = (out[i] + cf * Lc[c]) % R
        return out

    u = wire_eval([(i, c, cf) for c, row in enumerate(arows) for i, cf in row] + [(i, nc + i, 1) for i in range(npub + 1)])
    v = wire_eval([(i, c, cf) for c, row in enumerate(brows) for i, cf in row])
    ww = wire_eval([(nin + c, c, 1) for c in range(nc)])
    g1 = g1_generator_mont().reshape(1, -1)
    g2 = g2_generator_mont().reshape(1, -1)
    m1 = lambda ks: o.scmul(ints_to_limbs(ks), g1, 0)  # noqa: E731
    m2 = lambda ks: o.scmul(ints_to_limbs(ks), g2, 1)  # noqa: E731
    dinv, ginv = pow(de, -1, R), pow(ga, -1, R)
    pk = {"n_vars": nv, "n_public": npub, "domain_size": m, "polsA": polsA, "polsB": polsB,
          "A": np.concatenate([m1(u), m1([al, de])]), "B1": np.concatenate([m1(v), m1([be, de])]),
          "B2": np.concatenate([m2(v), m2([be, de])]),
          "C": m1([(be * u[i] + al * v[i] + ww[i]) * dinv % R for i in range(nv)]),
          "hExps": m1([pow(t, j, R) * (pow(t, m, R) - 1) * dinv % R for j in range(m - 1)]),
          "delta_1": m1([de])[0]}
    vk = {"alpha_1": m1([al])[0], "beta_2": m2([be])[0], "gamma_2": m2([ga])[0], "delta_2": m2([de])[0],
          "IC": m1([(be * u[i] + al * v[i] + ww[i]) * ginv % R for i in range(npub + 1)])}
    return pk, vk, ints_to_limbs(w)


def test_cpu_prover_proof_verifies(oracle):
    pk, vk, w = _tiny_groth(oracle)
    proof = cpu_prove(oracle, pk, w, 12345, 67890)
    assert verify(vk, proof, w[1:2])
    bad = w[1:2].copy()
    bad[0, 1] ^= 4
    assert not verify(vk, proof, bad)


def test_cpu_prover_reference_library_identical(oracle, reflib):
    pk, vk, w = _tiny_groth(oracle, L=5, seed=9)
    assert np.array_equal(cpu_prove(oracle, pk, w, 777, 888), cpu_prove(oracle, pk, w, 777, 888, ref=reflib))


def test_cpu_builder_key_matches_integer_setup(oracle):
    """oracle/synth_cpu.py (the builder bench.py's reference arm uses) against Groth16 setup
    restated with Python integers and the oracle's double-and-add scalar multiplication, on
    the benchmark circuit family at m = 2^5; its witness satisfies every constraint and its
    proof, from the staged CPU sequence, verifies."""
    from oracle.oracle import from_mont_int
    from oracle.prover import cpu_prove_stages
    from oracle.synth_cpu import CpuCircuit, cpu_setup_pk
    from cusnarks_b200.groth import toxic_waste
    L = 5
    c = CpuCircuit(oracle, L, seed=21, n_public=2)
    m, nv, nc = c.m, c.n_vars, c.n_constraints
    w = [limbs_to_int(x) for x in c.w]
    mi = pow(1 << 256, -1, R)
    coef = lambda x: limbs_to_int(x) * mi % R  # noqa: E731
    for k in range(nc):
        a = sum(coef(c.a_coeff[k, j]) * w[c.a_wire[k, j]] for j in range(3)) % R
        b = sum(coef(c.b_coeff[k, j]) * w[c.b_wire[k, j]] for j in range(3)) % R
        assert a * b % R == w[c.n_inputs + k]
    pk = cpu_setup_pk(oracle, c, seed=22)
    t, al, be, ga, de = toxic_waste(22)
    omega = from_mont_int(limbs_to_int(oracle.find_roots(L)[1]), 1)
    Lc = [pow(omega, i, R) * (pow(t, m, R) - 1) * pow(m * (t - pow(omega, i, R)), -1, R) % R for i in range(m)]

    def wire_eval(pol):
        out, off = [0] * nv, 1 + nv
        for i in range(nv):
            cnt = int(pol[1 + i])
            for j in range(cnt):
                row = int(pol[off + j])
                out[i] = (out[i] + coef(pol[off + cnt + 8 * j:off + cnt + 8 * j + 8]) * Lc[row]) % R
            off += 9 * cnt
        return out

    u, v, ww = (wire_eval(p) for p in (c.polsA, c.polsB, c.polsC))
    g1 = g1_generator_mont().reshape(1, -1)
    g2 = g2_generator_mont().reshape(1, -1)
    m1 = lambda ks: oracle.scmul(ints_to_limbs(ks), g1, 0)  # noqa: E731
    m2 = lambda ks: oracle.scmul(ints_to_limbs(ks), g2, 1)  # noqa: E731
    dinv = pow(de, -1, R)
    assert np.array_equal(pk["A"], np.concatenate([m1(u), m1([al, de])]))
    assert np.array_equal(pk["B1"], np.concatenate([m1(v), m1([be, de])]))
    assert np.array_equal(pk["B2"], np.concatenate([m2(v), m2([be, de])]))
    assert np.array_equal(pk["C"], m1([(be * u[i] + al * v[i] + ww[i]) * dinv % R for i in range(nv)]))
    assert np.array_equal(pk["hExps"], m1([pow(t, j, R) * (pow(t, m, R) - 1) * dinv % R for j in range(m - 1)]))
    ginv = pow(ga, -1, R)
    assert np.array_equal(pk["vk"]["IC"], m1([(be * u[i] + al * v[i] + ww[i]) * ginv % R for i in range(3)]))
    stages, st = cpu_prove_stages(oracle, pk, c.w, 4242, 2424)
    assert [n for n, _ in stages] == ["qap", "hstep", "msm_A", "msm_B2", "msm_B1", "msm_C", "msm_H+combine"]
    for _, fn in stages:
        fn()
    assert np.array_equal(st["proof"], cpu_prove(oracle, pk, c.w, 4242, 2424))
    assert verify(pk["vk"], st["proof"], c.public_inputs)
