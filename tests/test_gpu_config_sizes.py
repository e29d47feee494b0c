"""Parity at the sizes the benchmark configurations name, against the oracle and the
reference's own CPU library (oracle/_ref), never GPU against GPU:

* config 1: one G1 MSM of 2^16 terms (ec_jacreduce_server_h, src/cuda/ec.cpp:1536);
* config 2: the native 2^20 NTT and INTT (ntt_h / intt_h, src/cuda/ntt.cpp:453 / :583) and
  the 2^20 H step, reference variant (interpol_and_mul_h, ntt.cpp:778) and coset variant;
* config 3: one proof of the 2^20-constraint benchmark circuit through cs_prove, byte for
  byte against the reference's CPU proving sequence (groth_prover.py:585-790, :1414-1453)
  run in the reference's library, plus the Groth16 pairing check (and its failure on a
  changed public input).  At this size the G2 MSM runs its batch-affine rounds over the
  fixed-base table and the G1 MSMs the throughput form of the bucket accumulation.
The CPU builder of the benchmark circuit and key (oracle/synth_cpu.py, which bench.py's
reference arm uses) is checked against the GPU builder word for word.  A 2^22-constraint proof
is checked by the pairing equation; proofs of 2^15 and 2^17 constraints and a generic G2 MSM of
2^15 terms (mid sizes, whose accumulation tasks are sized to the GPU) against the CPU.
"""
import numpy as np
import pytest

from oracle.oracle import random_field, ints_to_limbs

pytestmark = pytest.mark.gpu

BENCH_R = 0x1234567890abcdef
BENCH_S = 0xfedcba0987654321


@pytest.fixture(scope="module")
def ctx():
    from cusnarks_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def test_config1_g1_msm_2e16(ctx, oracle):
    """Seeded scalars uniform in Fr and bases k_i G1 (k_i seeded, made on the CPU): the GPU
    MSM (host and device entry points) equals the oracle and the reference library."""
    import torch
    from oracle.oracle import RefLib
    from oracle.synth_cpu import fixed_base_mul
    n = 1 << 16
    rng = np.random.Generator(np.random.PCG64(16))
    k = random_field(rng, n, 1)
    s = random_field(rng, n, 1)
    pts = fixed_base_mul(oracle, k)
    want = oracle.msm(s, pts)
    if RefLib.available():
        assert np.array_equal(RefLib.get().msm(s, pts, 0, 6), want)
    assert np.array_equal(ctx.msm(s, pts), want)
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    ds, dp = _dev(s), _dev(pts)
    ctx.msm_device(ds.data_ptr(), dp.data_ptr(), n, out.data_ptr())
    ctx.sync()
    assert np.array_equal(_host(out), want)


def test_config2_ntt_intt_2e20(ctx, oracle):
    import torch
    L = 20
    rng = np.random.Generator(np.random.PCG64(220))
    A = oracle.to_mont(random_field(rng, 1 << L, 1), 1)
    roots = oracle.find_roots(L)
    dA = _dev(A)
    dF, dB, dN = torch.empty_like(dA), torch.empty_like(dA), torch.empty_like(dA)
    ctx.ntt_device(dA.data_ptr(), dF.data_ptr(), L, 1)
    ctx.ntt_device(dF.data_ptr(), dB.data_ptr(), L, -1, fmat=1)
    ctx.ntt_device(dA.data_ptr(), dN.data_ptr(), L, -1, fmat=0)
    ctx.sync()
    F = oracle.ntt(A, roots, L, 1, 1, 1, 1)
    assert np.array_equal(_host(dF), F)
    assert np.array_equal(_host(dB), oracle.intt(F, roots, L, 1, 1, 1))
    assert np.array_equal(_host(dB), A)
    assert np.array_equal(_host(dN), oracle.intt(A, roots, L, 1, 0, 1))


def test_config2_hstep_2e20_both_variants(ctx, oracle):
    import ctypes
    import torch
    from oracle.oracle import _p
    L = 20
    m = 1 << L
    rng = np.random.Generator(np.random.PCG64(221))
    A = oracle.to_mont(random_field(rng, m, 1), 1)
    B = oracle.to_mont(random_field(rng, m, 1), 1)
    C = oracle.to_mont(random_field(rng, m, 1), 1)
    dA, dB, dC = _dev(A), _dev(B), _dev(C)
    dM = torch.zeros((2 * m, 8), dtype=torch.int32, device="cuda")
    dH = torch.zeros((m, 8), dtype=torch.int32, device="cuda")
    ctx.hstep_device(0, dA.data_ptr(), dB.data_ptr(), 0, L, dM.data_ptr())
    ctx.hstep_device(1, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), L, dH.data_ptr())
    ctx.sync()
    M = _host(dM)
    assert np.array_equal(M, oracle.interpolandmul(A, B, oracle.find_roots(L + 1), L, 2))
    assert np.array_equal(_host(dH), oracle.hstep_coset(A, B, C, L))
    # A*B - C vanishing on the domain: the coset quotient equals the reference variant's
    # upper half (the Groth16 H polynomial)
    AB = np.zeros_like(A)
    oracle.lib.or_montmult_batch(_p(AB), _p(A), _p(B), ctypes.c_uint64(m), 1)
    dAB = _dev(AB)
    ctx.hstep_device(1, dA.data_ptr(), dB.data_ptr(), dAB.data_ptr(), L, dH.data_ptr())
    ctx.sync()
    H = _host(dH)
    assert np.array_equal(H[:m - 1], M[m:2 * m - 1]) and not H[m - 1].any()


@pytest.fixture(scope="module")
def bench_case(ctx):
    """The benchmark's 2^20-constraint circuit and key (seeds of bench.py's rank 0)."""
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, pk_to_host
    circ = SyntheticCircuit(ctx, 20, seed=100)
    pk = setup_pk(ctx, circ, seed=101)
    return circ, pk, pk_to_host(pk)


def test_config3_cpu_builder_equals_gpu_builder(oracle, bench_case):
    """bench.py's reference arm builds the 2^20 circuit and key on the CPU: the same words as
    the GPU builder, so both arms prove the same statement with the same key."""
    from oracle.synth_cpu import CpuCircuit, cpu_setup_pk
    circ, _, host = bench_case
    cc = CpuCircuit(oracle, 20, seed=100)
    assert np.array_equal(cc.w, circ.w)
    for k in ("polsA", "polsB", "polsC"):
        assert np.array_equal(getattr(cc, k), getattr(circ, k)), k
    cpk = cpu_setup_pk(oracle, cc, seed=101)
    for k in ("A", "B1", "B2", "C", "hExps", "delta_1", "polsA", "polsB"):
        assert np.array_equal(np.asarray(cpk[k]).reshape(-1), np.asarray(host[k]).reshape(-1)), k
    for k, v in cpk["vk"].items():
        assert np.array_equal(np.asarray(v).reshape(-1), np.asarray(host["vk"][k]).reshape(-1)), k


def test_config3_prove_2e20_matches_reference_and_verifies(ctx, oracle, bench_case):
    import torch
    from cusnarks_b200.groth import Prover
    from oracle.oracle import RefLib
    from oracle.prover import cpu_prove, verify
    circ, pk, host = bench_case
    prover = Prover(ctx, pk)
    try:
        assert all(c > 0 for c in prover.fixed_windows())
        r, s = ints_to_limbs([BENCH_R])[0], ints_to_limbs([BENCH_S])[0]
        proof = prover.prove(circ.w, r, s)
        d_proof = torch.zeros(64, dtype=torch.int32, device="cuda")
        prover.prove_device(circ.d_w.data_ptr(), r, s, d_proof.data_ptr())
        ctx.sync()
        assert np.array_equal(_host(d_proof), proof)
    finally:
        prover.close()
    ref = RefLib.get() if RefLib.available() else None
    want = cpu_prove(oracle, host, circ.w, BENCH_R, BENCH_S, ref=ref)
    assert np.array_equal(proof, want)
    assert verify(host["vk"], proof, circ.public_inputs)
    bad = circ.public_inputs.copy()
    bad[0, 0] ^= 1
    assert not verify(host["vk"], proof, bad)


def test_prove_2e22_verifies(ctx):
    """The 2^22-constraint proof the reference publishes a time for (its README: 18 s on two
    GTX 1080): proved with resident fixed-base tables (G1 window 20; the G2 MSM with its
    batch-affine rounds), the host and device entry points agree, the Groth16 pairing check
    passes and fails on a changed public input.  (Byte parity with the CPU sequence is checked
    at 2^20 above; the CPU sequence at 2^22 takes minutes.)"""
    import torch
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, Prover
    from oracle.prover import verify
    circ = SyntheticCircuit(ctx, 22, seed=122)
    pk = setup_pk(ctx, circ, seed=123)
    prover = Prover(ctx, pk)
    try:
        r, s = ints_to_limbs([BENCH_R])[0], ints_to_limbs([BENCH_S])[0]
        proof = prover.prove(circ.w, r, s)
        d_proof = torch.zeros(64, dtype=torch.int32, device="cuda")
        prover.prove_device(circ.d_w.data_ptr(), r, s, d_proof.data_ptr())
        ctx.sync()
        assert np.array_equal(_host(d_proof), proof)
    finally:
        prover.close()
    assert verify(pk["vk"], proof, circ.public_inputs)
    bad = circ.public_inputs.copy()
    bad[0, 0] ^= 1
    assert not verify(pk["vk"], proof, bad)


@pytest.mark.parametrize("log_m", [15, 17])
def test_prove_mid_sizes_match_cpu(ctx, oracle, log_m):
    """Proofs of 2^15 and 2^17 constraints, where the MSMs are too large for the latency form
    and too small to fill the GPU at full-length tasks (their accumulation tasks are sized to
    the GPU): byte for byte the CPU proving sequence (the reference library where built),
    and the pairing check."""
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, pk_to_host, Prover
    from oracle.oracle import RefLib
    from oracle.prover import cpu_prove, verify
    circ = SyntheticCircuit(ctx, log_m, seed=130 + log_m)
    pk = setup_pk(ctx, circ, seed=131 + log_m)
    host = pk_to_host(pk)
    prover = Prover(ctx, pk)
    try:
        proof = prover.prove(circ.w, ints_to_limbs([BENCH_R])[0], ints_to_limbs([BENCH_S])[0])
    finally:
        prover.close()
    ref = RefLib.get() if RefLib.available() else None
    assert np.array_equal(proof, cpu_prove(oracle, host, circ.w, BENCH_R, BENCH_S, ref=ref))
    assert verify(host["vk"], proof, circ.public_inputs)


def test_g2_generic_msm_2e15(ctx, oracle):
    """A generic (no table) G2 MSM of 2^15 terms, a mid size whose accumulation tasks are sized
    to the GPU: equal to the oracle (and the reference library where built)."""
    from oracle.oracle import RefLib
    from oracle.synth_cpu import fixed_base_mul
    n = 1 << 15
    rng = np.random.Generator(np.random.PCG64(315))
    pts = fixed_base_mul(oracle, random_field(rng, n, 1), ec2=True)
    s = random_field(rng, n, 1)
    want = oracle.msm(s, pts, ec2=1)
    if RefLib.available():
        assert np.array_equal(RefLib.get().msm(s, pts, 1, 6), want)
    assert np.array_equal(ctx.msm(s, pts, ec2=True), want)
