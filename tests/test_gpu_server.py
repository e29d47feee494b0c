"""Served proving: proofs made in a concurrent mix of circuits equal the proofs made alone
(byte for byte); admission by device memory refuses a request that can never fit."""
import numpy as np
import pytest

from oracle.oracle import ints_to_limbs, R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from cusnarks_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def keys(ctx):
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, Prover
    out = []
    for log_m, seed in ((7, 21), (9, 22), (11, 23)):
        circ = SyntheticCircuit(ctx, log_m, seed=seed)
        pk = setup_pk(ctx, circ, seed=seed + 1)
        out.append((circ, pk, Prover(ctx, pk)))
    yield out
    for _, _, p in out:
        p.close()


def _rs(i):
    r = (0x1234567 * (i + 3) + 99991) % R
    s = (0x7654321 * (i + 5) + 77773) % R
    return ints_to_limbs([r])[0], ints_to_limbs([s])[0]


def test_mix_equals_alone(keys):
    from cusnarks_b200.server import ProveServer
    jobs = [(i % 3 if i % 4 else 2, i) for i in range(14)]   # uneven mix, the largest most
    alone = {}
    for k, i in jobs:
        circ, _, prover = keys[k]
        r, s = _rs(i)
        alone[i] = prover.prove(circ.w, r, s)
    srv = ProveServer(0, slots=3, reserve_bytes=64 << 20)
    try:
        kid = [srv.add_key(p) for _, _, p in keys]
        tickets = []
        for k, i in jobs:
            r, s = _rs(i)
            tickets.append((i, srv.submit(kid[k], keys[k][0].w, r, s)))
        for i, t in tickets:
            proof, info = srv.wait(t, timeout=120.0)
            assert np.array_equal(proof, alone[i]), i
            assert info["latency_ms"] >= info["queue_ms"] >= 0.0
        st = srv.stats()
        assert st["completed"] == len(jobs) and st["failed"] == 0 and st["queued"] == 0
        assert st["max_concurrent"] >= 2
    finally:
        srv.close()


def test_admission_refuses_what_cannot_fit(keys):
    """A reserve larger than the device: with nothing running, the request is refused
    with CS_ERR_NOMEM (no allocation is attempted)."""
    from cusnarks_b200.server import ProveServer
    from cusnarks_b200._lib import CsError, CS_ERR_NOMEM
    srv = ProveServer(0, slots=2, reserve_bytes=1 << 50)
    try:
        k = srv.add_key(keys[0][2])
        r, s = _rs(0)
        t = srv.submit(k, keys[0][0].w, r, s)
        with pytest.raises(CsError) as ei:
            srv.wait(t, timeout=60.0)
        assert ei.value.code == CS_ERR_NOMEM
        assert srv.stats()["rejected"] == 1
    finally:
        srv.close()


def test_same_key_batches_equal_alone(keys):
    """One slot, a request of the 2^11 key first (it grows the slot's scratch while the rest
    queue), then 13 requests of the 2^7 key with distinct witnesses and (r, s): the slot
    proves the queued ones in same-key batches (8, then 4, then 1) and every proof equals
    the lone proof of its own witness and (r, s)."""
    from cusnarks_b200.server import ProveServer
    rng = np.random.Generator(np.random.PCG64(77))
    circ0, _, prover0 = keys[0]
    circ2, _, prover2 = keys[2]
    ws = []
    for i in range(13):
        w = circ0.w.copy()
        lo = circ0.n_public + 1
        w[lo:lo + 4] = ints_to_limbs([int(x) % R for x in rng.integers(1, 1 << 62, 4)])
        ws.append(w)
    alone = [prover0.prove(ws[i], *_rs(i)) for i in range(13)]
    first = prover2.prove(circ2.w, *_rs(99))
    srv = ProveServer(0, slots=1, reserve_bytes=64 << 20, max_batch=8)
    try:
        k0, k2 = srv.add_key(prover0), srv.add_key(prover2)
        t_first = srv.submit(k2, circ2.w, *_rs(99))
        tickets = [srv.submit(k0, ws[i], *_rs(i)) for i in range(13)]
        assert np.array_equal(srv.wait(t_first, timeout=120.0)[0], first)
        for i, t in enumerate(tickets):
            proof, _ = srv.wait(t, timeout=120.0)
            assert np.array_equal(proof, alone[i]), i
        st = srv.stats()
        assert st["completed"] == 14 and st["failed"] == 0
        assert st["batches"] >= 1 and 4 <= st["max_batch_seen"] <= 8, st
    finally:
        srv.close()


def test_key_added_while_serving(keys):
    """Slots size themselves for the keys registered when they first take work; a larger key
    added later makes them grow once more.  Proofs before and after equal the lone proofs."""
    from cusnarks_b200.server import ProveServer
    (c0, _, p0), (c2, _, p2) = keys[0], keys[2]
    alone0 = [p0.prove(c0.w, *_rs(i)) for i in range(6)]
    alone2 = [p2.prove(c2.w, *_rs(50 + i)) for i in range(6)]
    srv = ProveServer(0, slots=2, reserve_bytes=64 << 20, max_batch=4)
    try:
        k0 = srv.add_key(p0)
        first = [srv.submit(k0, c0.w, *_rs(i)) for i in range(6)]
        for i, t in enumerate(first):
            assert np.array_equal(srv.wait(t, timeout=120.0)[0], alone0[i]), i
        k2 = srv.add_key(p2)
        mixed = []
        for i in range(6):
            mixed.append((alone2[i], srv.submit(k2, c2.w, *_rs(50 + i))))
            mixed.append((alone0[i], srv.submit(k0, c0.w, *_rs(i))))
        for want, t in mixed:
            assert np.array_equal(srv.wait(t, timeout=120.0)[0], want)
        st = srv.stats()
        assert st["completed"] == 18 and st["failed"] == 0
    finally:
        srv.close()
