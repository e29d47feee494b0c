"""Failures on the host side, none on the GPU: an injected device-allocation failure is
reported as CS_ERR_NOMEM and the context stays usable (the next call is correct); queued
server requests can be cancelled; a missing witness file is recorded as a failed request."""
import time

import numpy as np
import pytest

from oracle.oracle import random_field, ints_to_limbs
from tests.gpu_common import random_points

pytestmark = pytest.mark.gpu


def test_alloc_failure_is_reported_and_recovered(oracle):
    from cusnarks_b200 import Context, lib
    from cusnarks_b200._lib import CsError, CS_ERR_NOMEM
    rng = np.random.Generator(np.random.PCG64(404))
    pts = random_points(oracle, rng, 512)
    s = random_field(rng, 512, 1)
    ctx = Context(0)               # fresh arenas: the first MSM must grow them
    try:
        lib().cs_debug_fail_allocs(1)
        with pytest.raises(CsError) as ei:
            ctx.msm(s, pts)
        assert ei.value.code == CS_ERR_NOMEM
        assert np.array_equal(ctx.msm(s, pts), oracle.msm(s, pts))
    finally:
        lib().cs_debug_fail_allocs(0)
        ctx.close()


def test_prove_alloc_failure_then_success():
    from cusnarks_b200 import Context, lib
    from cusnarks_b200._lib import CsError, CS_ERR_NOMEM
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, Prover
    ctx = Context(0)
    circ = SyntheticCircuit(ctx, 8, seed=81)
    pk = setup_pk(ctx, circ, seed=82)
    r, s = ints_to_limbs([11])[0], ints_to_limbs([13])[0]
    ref = Prover(ctx, pk)
    want = ref.prove(circ.w, r, s)
    ref.close()
    ctx2 = Context(0)              # fresh context: the proof's scratch must be allocated
    p2 = Prover(ctx2, pk)
    try:
        lib().cs_debug_fail_allocs(1)
        with pytest.raises(CsError) as ei:
            p2.prove(circ.w, r, s)
        assert ei.value.code == CS_ERR_NOMEM
        assert np.array_equal(p2.prove(circ.w, r, s), want)
    finally:
        lib().cs_debug_fail_allocs(0)
        p2.close()
        ctx2.close()
        ctx.close()


def test_server_cancel_and_stats():
    from cusnarks_b200 import Context
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, Prover
    from cusnarks_b200.server import ProveServer
    from cusnarks_b200._lib import CsError, CS_ERR_CANCELLED
    ctx = Context(0)
    circ = SyntheticCircuit(ctx, 12, seed=91)
    prover = Prover(ctx, setup_pk(ctx, circ, seed=92))
    r, s = ints_to_limbs([5])[0], ints_to_limbs([7])[0]
    want = prover.prove(circ.w, r, s)
    srv = ProveServer(0, slots=1, reserve_bytes=0)
    try:
        k = srv.add_key(prover)
        tickets = [srv.submit(k, circ.w, r, s) for _ in range(6)]
        cancelled = [t for t in tickets[3:] if srv.cancel(t)]
        assert cancelled, "no queued request left to cancel"
        for t in tickets:
            if t in cancelled:
                with pytest.raises(CsError) as ei:
                    srv.wait(t, timeout=60.0)
                assert ei.value.code == CS_ERR_CANCELLED
            else:
                proof, _ = srv.wait(t, timeout=60.0)
                assert np.array_equal(proof, want)
        st = srv.stats()
        assert st["cancelled"] == len(cancelled) and st["completed"] == 6 - len(cancelled)
        assert 0.0 < st["p50_ms"] <= st["p99_ms"] and st["hbm_total_bytes"] > st["hbm_free_bytes"] > 0
        assert not srv.cancel(tickets[0])      # finished: not cancellable
    finally:
        srv.close()
        prover.close()
        ctx.close()


def test_netserver_missing_witness(tmp_path):
    from cusnarks_b200 import Context
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, Prover
    from cusnarks_b200.netserver import NetProveServer, request
    ctx = Context(0)
    circ = SyntheticCircuit(ctx, 6, seed=95)
    prover = Prover(ctx, setup_pk(ctx, circ, seed=96))
    srv = NetProveServer(prover, circ.n_public, port=0, slots=1)
    try:
        request(srv.port, {"witness_f": str(tmp_path / "nope.bin"), "proof_f": str(tmp_path / "p.json"),
                           "public_data_f": str(tmp_path / "q.json"), "verify_en": 0}, reply=False)
        deadline = time.time() + 30
        while True:
            rec = request(srv.port, {"list": 0})
            if rec and rec["result"] != -1:
                break
            assert time.time() < deadline
            time.sleep(0.05)
        assert rec["result"] == 0 and "error" in rec
        assert request(srv.port, {"is_alive": 1}) == {"status": 1}   # still serving
    finally:
        try:
            request(srv.port, {"stop_server": 1}, reply=False)
        except OSError:
            pass
        srv.close()
        prover.close()
        ctx.close()


def test_prover_without_room_for_tables_proves_generically():
    """Automatic fixed-base tables that cannot be allocated (injected failure) leave the key
    without tables; the proofs then run the generic MSM and are the same bytes."""
    from cusnarks_b200 import Context, lib
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, Prover
    ctx = Context(0)
    circ = SyntheticCircuit(ctx, 8, seed=91)
    pk = setup_pk(ctx, circ, seed=92)
    r, s = ints_to_limbs([17])[0], ints_to_limbs([19])[0]
    ref = Prover(ctx, pk)
    assert ref.fixed_windows()[0] > 0 and ref.fixed_base_note is None
    want = ref.prove(circ.w, r, s)
    ref.close()
    ctx2 = Context(0)              # fresh arenas: the table build must allocate scratch
    try:
        lib().cs_debug_fail_allocs(1)
        p2 = Prover(ctx2, pk)
        lib().cs_debug_fail_allocs(0)
        assert p2.fixed_windows() == [0, 0, 0, 0, 0] and p2.fixed_base_note
        assert np.array_equal(p2.prove(circ.w, r, s), want)
        p2.close()
    finally:
        lib().cs_debug_fail_allocs(0)
        ctx2.close()
        ctx.close()
