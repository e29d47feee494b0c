"""Proving-key and witness files: the loader reads a key written by the reference's own writer
(pysnarks_utils.pkvars_to_bin, FMT_MONT, affine, extended) and a witness written by the
reference's writeWitnessFile_h; the writers reproduce those files word for word."""
import json

import numpy as np

from cusnarks_b200 import pkfile


def _inputs(golden):
    return golden("pk_files.npz")


def test_read_reference_pk_bin(golden):
    g = _inputs(golden)
    pk = pkfile.read_pk_bin(g["pk_bin"])
    nv, m = int(g["n_vars"]), int(g["domain"])
    assert (pk["n_vars"], pk["n_public"], pk["domain_size"]) == (nv, int(g["n_public"]), m)
    assert np.array_equal(pk["A"], np.concatenate([g["A"], g["alfa_1"], g["delta_1"]]))
    assert np.array_equal(pk["B1"], np.concatenate([g["B1"], g["beta_1"], g["delta_1"]]))
    assert np.array_equal(pk["B2"], np.concatenate([g["B2"], g["beta_2"], g["delta_2"]]))
    assert np.array_equal(pk["C"], g["C"])
    assert np.array_equal(pk["hExps"], g["hExps"][:m - 1])
    assert np.array_equal(pk["delta_1"], g["delta_1"].reshape(1, 16))
    for k in ("polsA", "polsB"):
        p = g[k].reshape(-1)
        assert np.array_equal(pk[k][:p.size], p)
        assert not pk[k][p.size:].any()          # the writer's zero padding to domain*8 words


def test_write_matches_reference_writer(golden):
    g = _inputs(golden)
    pk = {"n_vars": int(g["n_vars"]), "n_public": int(g["n_public"]), "domain_size": int(g["domain"]),
          "polsA": g["polsA"], "polsB": g["polsB"],
          "A": np.concatenate([g["A"], g["alfa_1"], g["delta_1"]]),
          "B1": np.concatenate([g["B1"], g["beta_1"], g["delta_1"]]),
          "B2": np.concatenate([g["B2"], g["beta_2"], g["delta_2"]]),
          "C": g["C"], "hExps": g["hExps"], "delta_1": g["delta_1"]}
    assert np.array_equal(pkfile.write_pk_bin(pk), g["pk_bin"])


def test_witness_files(golden, tmp_path):
    g = _inputs(golden)
    w, nv = g["witness"], int(g["n_vars"])
    assert np.array_equal(pkfile.write_witness_bin(w), g["witness_bin"])
    p = tmp_path / "w.bin"
    g["witness_bin"].astype("<u4").tofile(p)
    assert np.array_equal(pkfile.read_witness(p, nv), w)
    ints = [sum(int(x) << (32 * i) for i, x in enumerate(row)) for row in w]
    (tmp_path / "w.json").write_text(json.dumps([str(v) for v in ints]))
    (tmp_path / "w.txt").write_text("\n".join(str(v) for v in ints) + "\n")
    assert np.array_equal(pkfile.read_witness(tmp_path / "w.json", nv), w)
    assert np.array_equal(pkfile.read_witness(tmp_path / "w.txt", nv), w)
    dat = np.concatenate([np.zeros(8, np.uint32), w.reshape(-1)])
    dat.astype("<u4").tofile(tmp_path / "w.dat")
    assert np.array_equal(pkfile.read_witness(tmp_path / "w.dat", nv), w)


def test_rejects_other_files(golden):
    g = _inputs(golden)
    bad = g["pk_bin"].copy()
    bad[1] = 7
    try:
        pkfile.read_pk_bin(bad)
    except ValueError:
        pass
    else:
        raise AssertionError("a non-proving-key file was accepted")


def test_proof_json_normal_form():
    """proof.json carries normal-form decimal coordinates (pi_a, pi_c with z = 1, pi_b with
    z = (1, 0)), as the reference's write_proof: the generators come out as their integers."""
    from cusnarks_b200 import netserver
    from tests.gpu_common import g1_generator_mont, g2_generator_mont
    from oracle.oracle import G1_GEN, G2_GEN
    proof = np.concatenate([g1_generator_mont(), g2_generator_mont(), g1_generator_mont()])
    j = netserver.proof_to_json(proof)
    assert j["pi_a"] == [str(G1_GEN[0]), str(G1_GEN[1]), "1"] == j["pi_c"]
    assert j["pi_b"] == [[str(G2_GEN[0][0]), str(G2_GEN[0][1])], [str(G2_GEN[1][0]), str(G2_GEN[1][1])], ["1", "0"]]
    assert j["protocol"] == "groth"


def test_truncated_files_are_rejected(golden, tmp_path):
    g = _inputs(golden)
    import pytest
    with pytest.raises(ValueError):
        pkfile.read_pk_bin(g["pk_bin"][:200])           # header only
    with pytest.raises(ValueError):
        pkfile.read_pk_bin(g["pk_bin"][:-500])          # points cut off
    p = tmp_path / "w.bin"
    g["witness_bin"][:40].astype("<u4").tofile(p)
    with pytest.raises(ValueError):
        pkfile.read_witness(p, int(g["n_vars"]))
