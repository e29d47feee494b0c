"""Keys and witnesses through the reference file formats on the GPU: a key written to the .bin
format and read back proves byte-identically; the reference-protocol TCP front end admits
concurrent requests and writes proofs that pass the pairing check."""
import json
import time

import numpy as np
import pytest

from oracle.oracle import ints_to_limbs
from oracle.prover import verify

pytestmark = pytest.mark.gpu

Q = 21888242871839275222246405745257275088696311157297823662689037894645226208583


@pytest.fixture(scope="module")
def ctx():
    from cusnarks_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def circuit(ctx):
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, pk_to_host
    circ = SyntheticCircuit(ctx, 8, seed=61)
    pk = setup_pk(ctx, circ, seed=62)
    return circ, pk, pk_to_host(pk)


def test_pk_bin_roundtrip_proves_identically(ctx, circuit, tmp_path):
    from cusnarks_b200 import pkfile
    from cusnarks_b200.groth import Prover
    circ, pk, host = circuit
    path = tmp_path / "pk.bin"
    pkfile.write_pk_bin(host, path)
    loaded = pkfile.read_pk_bin(path)
    r, s = ints_to_limbs([123456789])[0], ints_to_limbs([987654321])[0]
    p1, p2 = Prover(ctx, pk), Prover(ctx, loaded)
    try:
        wpath = tmp_path / "w.bin"
        pkfile.write_witness_bin(circ.w, wpath)
        w = pkfile.read_witness(wpath, circ.n_vars)
        assert np.array_equal(p2.prove(w, r, s), p1.prove(circ.w, r, s))
    finally:
        p1.close()
        p2.close()


def _mont_words(vals):
    return ints_to_limbs([(int(v) << 256) % Q for v in vals]).reshape(-1)


def test_reference_protocol_server(ctx, circuit, tmp_path):
    from cusnarks_b200 import pkfile
    from cusnarks_b200.groth import Prover
    from cusnarks_b200.netserver import NetProveServer, request
    circ, pk, host = circuit
    prover = Prover(ctx, pk)
    srv = NetProveServer(prover, circ.n_public, port=0, slots=2)
    try:
        assert request(srv.port, {"is_alive": 1}) == {"status": 1}
        wpath = tmp_path / "w.bin"
        pkfile.write_witness_bin(circ.w, wpath)
        outs = []
        for k in range(3):
            pf = tmp_path / f"proof{k}.json"
            qf = tmp_path / f"public{k}.json"
            request(srv.port, {"witness_f": str(wpath), "proof_f": str(pf), "public_data_f": str(qf),
                               "verify_en": 0}, reply=False)
            outs.append((pf, qf))
        deadline = time.time() + 120
        recs = []
        for k in range(3):
            while True:
                rec = request(srv.port, {"list": k})
                if rec and rec["result"] != -1:
                    break
                assert time.time() < deadline, "proof not done in time"
                time.sleep(0.05)
            recs.append(rec)
        assert [r["result"] for r in recs] == [1, 1, 1] and [r["proof_id"] for r in recs] == [0, 1, 2]
        for pf, qf in outs:
            j = json.loads(pf.read_text())
            proof = np.concatenate([_mont_words(j["pi_a"][:2]),
                                    _mont_words([j["pi_b"][0][0], j["pi_b"][0][1], j["pi_b"][1][0], j["pi_b"][1][1]]),
                                    _mont_words(j["pi_c"][:2])])
            pub = json.loads(qf.read_text())
            assert [int(x) for x in pub] == [sum(int(v) << (32 * i) for i, v in enumerate(row))
                                             for row in circ.public_inputs]
            assert verify(host["vk"], proof, circ.public_inputs)
    finally:
        try:
            request(srv.port, {"stop_server": 1}, reply=False)
        except OSError:
            pass
        srv.close()
        prover.close()
