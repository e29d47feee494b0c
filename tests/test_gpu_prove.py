"""GPU Groth16 prover: byte-identical to the CPU restatement of the reference's proving
sequence on the same key, witness, r and s, and every proof passes the pairing check."""
import numpy as np
import pytest

from oracle.oracle import ints_to_limbs, R
from oracle.prover import cpu_prove, verify

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from cusnarks_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _satisfied(circ, rows=64):
    from oracle.oracle import limbs_to_int
    w = [limbs_to_int(x) for x in circ.w]
    mont_inv = pow(1 << 256, -1, R)
    for c in range(min(rows, circ.n_constraints)):
        a = sum(limbs_to_int(circ.a_coeff[c, k]) * mont_inv * w[circ.a_wire[c, k]] for k in range(3)) % R
        b = sum(limbs_to_int(circ.b_coeff[c, k]) * mont_inv * w[circ.b_wire[c, k]] for k in range(3)) % R
        if a * b % R != w[circ.n_inputs + c]:
            return False
    return True


@pytest.mark.parametrize("log_m,seed", [(6, 3), (10, 11)])
def test_prove_matches_cpu_and_verifies(ctx, oracle, log_m, seed):
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, pk_to_host, Prover
    circ = SyntheticCircuit(ctx, log_m, seed=seed)
    assert _satisfied(circ)
    pk = setup_pk(ctx, circ, seed=seed + 1)
    prover = Prover(ctx, pk)
    rng = np.random.Generator(np.random.PCG64(seed + 2))
    r = int(rng.integers(1, 1 << 62)) * 1234567 % R
    s = int(rng.integers(1, 1 << 62)) * 7654321 % R
    proof = prover.prove(circ.w, ints_to_limbs([r])[0], ints_to_limbs([s])[0])
    host = pk_to_host(pk)
    want = cpu_prove(oracle, host, circ.w, r, s)
    assert np.array_equal(proof, want)
    assert verify(host["vk"], proof, circ.public_inputs)
    # a wrong public input must not verify
    bad = circ.public_inputs.copy()
    bad[0, 0] ^= 1
    assert not verify(host["vk"], proof, bad)
    # the default key holds fixed-base tables for all five MSMs
    assert all(c > 0 for c in prover.fixed_windows())
    # the same key uploaded from host memory, without tables (generic MSMs), gives the
    # same proof; proofs repeat; tables rebuilt with another window give it again
    prover2 = Prover(ctx, host, fixed_base=-1)
    assert prover2.fixed_windows() == [0] * 5
    assert np.array_equal(prover2.prove(circ.w, ints_to_limbs([r])[0], ints_to_limbs([s])[0]), proof)
    assert np.array_equal(prover.prove(circ.w, ints_to_limbs([r])[0], ints_to_limbs([s])[0]), proof)
    prover2.set_fixed_base(7)
    assert prover2.fixed_windows() == [7] * 5
    assert np.array_equal(prover2.prove(circ.w, ints_to_limbs([r])[0], ints_to_limbs([s])[0]), proof)
    prover.close(); prover2.close()


@pytest.mark.parametrize("log_m,n_public,seed", [(3, 1, 71), (4, 2, 72), (7, 3, 73), (8, 5, 74)])
def test_prove_public_inputs_and_tiny_domains(ctx, oracle, log_m, n_public, seed):
    """Several public inputs (the extra rows polsA gets) and domains down to 8 points: byte
    equal to the CPU sequence, verifies, and a changed public input fails."""
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, pk_to_host, Prover
    circ = SyntheticCircuit(ctx, log_m, seed=seed, n_public=n_public)
    pk = setup_pk(ctx, circ, seed=seed + 1)
    host = pk_to_host(pk)
    r, s = (seed * 1000003) % R, (seed * 999983 + 7) % R
    for fixed in (0, -1):
        prover = Prover(ctx, pk, fixed_base=fixed)
        proof = prover.prove(circ.w, ints_to_limbs([r])[0], ints_to_limbs([s])[0])
        prover.close()
        assert np.array_equal(proof, cpu_prove(oracle, host, circ.w, r, s)), fixed
    assert verify(host["vk"], proof, circ.public_inputs)
    bad = circ.public_inputs.copy()
    bad[-1, 0] ^= 1
    assert not verify(host["vk"], proof, bad)


def test_plain_per_call_path_matches(ctx):
    """The reference's flow through the drop-in entry points (one host-memory call per
    step, key re-sent per MSM) gives the resident prover's proof byte for byte."""
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, pk_to_host, Prover
    from cusnarks_b200.plain import PlainProver
    circ = SyntheticCircuit(ctx, 9, seed=41)
    pk = setup_pk(ctx, circ, seed=42)
    host = pk_to_host(pk)
    r, s = 0x1111111122222222333 % R, 0x44444444555555556666 % R
    want = Prover(ctx, pk).prove(circ.w, ints_to_limbs([r])[0], ints_to_limbs([s])[0])
    got = PlainProver(host).prove(circ.w, r, s)
    assert np.array_equal(got, want)


def test_dropin_mpoly_eval_fixture(golden):
    """mpoly_eval_server_h through the C ABI reproduces the reference library's output."""
    import ctypes
    from cusnarks_b200 import lib
    from cusnarks_b200._lib import MpolyEval
    f = golden("ref_transforms.npz")
    L = lib()
    for nv in (16, 300):
        nc = int(f[f"mpoly_ncons_{nv}"][0])
        pin = np.ascontiguousarray(f[f"mpoly_pin_{nv}"])
        w = np.ascontiguousarray(f[f"mpoly_w_{nv}"])
        out = np.zeros((nc, 8), np.uint32)
        a = MpolyEval(out.ctypes.data, w.ctypes.data, pin.ctypes.data, 0, 0, nv, 0, 0, 1)
        L.mpoly_eval_server_h(ctypes.byref(a))
        assert L.cs_qap_last_status() == 0
        assert np.array_equal(out, f[f"mpoly_out_{nv}"])


def test_prove_graph_replays_match_cpu(ctx, oracle):
    """The proof's launch sequence is captured as a CUDA graph on the first proof with a key,
    witness buffer and scratch, then replayed: replays with new r, s and a new witness in the
    same buffer give the CPU sequence's bytes; rebuilt tables and graphs turned off too."""
    import pytest as _pt
    from cusnarks_b200._lib import CsError
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, pk_to_host, Prover
    from oracle.oracle import random_field
    circ = SyntheticCircuit(ctx, 9, seed=91)
    pk = setup_pk(ctx, circ, seed=92)
    host = pk_to_host(pk)
    prover = Prover(ctx, pk)
    lim = lambda x: ints_to_limbs([x])[0]  # noqa: E731
    try:
        cases = [(circ.w, 11, 22), (circ.w, 11, 22), (circ.w, 333333, 4444)]
        w2 = random_field(np.random.Generator(np.random.PCG64(93)), circ.n_vars, 1)
        w2[0] = ints_to_limbs([1])[0]
        cases.append((w2, 55, 66))
        for w, r, s in cases:  # capture, replay, replay with new scalars, new witness
            got = prover.prove(w, lim(r), lim(s))
            assert np.array_equal(got, cpu_prove(oracle, host, w, r, s)), (r, s)
        with _pt.raises(CsError):
            prover.stages()  # the last proof was a replay: no stage events
        prover.set_fixed_base(7)  # tables move: the old graph must not be replayed
        assert np.array_equal(prover.prove(w2, lim(55), lim(66)), cpu_prove(oracle, host, w2, 55, 66))
        assert np.array_equal(prover.prove(circ.w, lim(11), lim(22)), cpu_prove(oracle, host, circ.w, 11, 22))
        ctx.set_prove_graphs(False)
        assert np.array_equal(prover.prove(circ.w, lim(11), lim(22)), cpu_prove(oracle, host, circ.w, 11, 22))
        assert prover.stages()["total"] > 0
    finally:
        ctx.set_prove_graphs(True)
        prover.close()


def test_prove_batch_matches_cpu(ctx, oracle):
    """cs_prove_batch_device: k proofs with one key in one pass (batched G1 / G2 / H MSMs over
    the fixed-base tables) give, proof by proof, the CPU sequence's bytes: a first call
    (captured), a replay with new witnesses and scalars, a different k, and a key without
    tables (proved one by one)."""
    import torch
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, pk_to_host, Prover
    from oracle.oracle import random_field
    circ = SyntheticCircuit(ctx, 8, seed=95)
    pk = setup_pk(ctx, circ, seed=96)
    host = pk_to_host(pk)
    rng = np.random.Generator(np.random.PCG64(97))

    def batch(prover, k):
        ws = [circ.w] + [random_field(rng, circ.n_vars, 1) for _ in range(k - 1)]
        for w in ws[1:]:
            w[0] = ints_to_limbs([1])[0]
        rs = [int(rng.integers(1, 1 << 62)) for _ in range(k)]
        ss = [int(rng.integers(1, 1 << 62)) * 3 % R for _ in range(k)]
        dws = [torch.from_numpy(np.ascontiguousarray(w).view(np.int32)).cuda() for w in ws]
        dp = torch.zeros((k, 64), dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        prover.prove_batch_device([t.data_ptr() for t in dws], [ints_to_limbs([x])[0] for x in rs],
                                  [ints_to_limbs([x])[0] for x in ss], [dp[i].data_ptr() for i in range(k)])
        ctx.sync()
        got = dp.cpu().numpy().view(np.uint32)
        for i in range(k):
            assert np.array_equal(got[i], cpu_prove(oracle, host, ws[i], rs[i], ss[i])), (k, i)

    prover = Prover(ctx, pk)
    try:
        batch(prover, 5)   # plan, capture, launch
        batch(prover, 5)   # replay with new inputs
        batch(prover, 3)
        batch(prover, 1)
    finally:
        prover.close()
    plain = Prover(ctx, pk, fixed_base=-1)
    try:
        batch(plain, 2)
    finally:
        plain.close()
