"""Host routines of the binding (no GPU): sortu256_idx_h and ntt_build_h against the
reference library's outputs, and the file routines on their documented layouts."""
import ctypes

import numpy as np

from cusnarks_b200 import lib, pkfile


def test_sortu256_idx_matches_reference(golden):
    g = golden("dropin.npz")
    v = np.ascontiguousarray(g["sort_v"])
    idx = np.zeros(v.shape[0], np.uint32)
    lib().sortu256_idx_h(idx.ctypes.data, v.ctypes.data, v.shape[0], 1)
    assert np.array_equal(idx, g["sort_idx"])
    lib().sortu256_idx_h(idx.ctypes.data, v.ctypes.data, v.shape[0], 0)
    assert np.array_equal(idx, np.arange(v.shape[0]))


def test_ntt_build_matches_reference(golden):
    g = golden("dropin.npz")
    for ns, want in zip(g["build_sizes"], g["build_params"]):
        buf = np.zeros(11, np.uint32)
        lib().ntt_build_h(buf.ctypes.data, int(ns))
        assert np.array_equal(buf, want), int(ns)


def test_file_routines(tmp_path):
    L = lib()
    rng = np.random.default_rng(5)
    data = rng.integers(0, 1 << 32, 64 * 8, dtype=np.uint64).astype(np.uint32)
    p = str(tmp_path / "d.bin").encode()
    L.writeU256DataFile_h(data.ctypes.data, p, data.size)
    L.appendU256DataFile_h(data.ctypes.data, p, 16)
    got = np.zeros(data.size + 16, np.uint32)
    L.readU256CircuitFile_h(got.ctypes.data, p, got.size)
    assert np.array_equal(got, np.concatenate([data, data[:16]]))
    part = np.zeros(40, np.uint32)
    L.readU256DataFileFromOffset_h(part.ctypes.data, p, 24, 40)
    assert np.array_equal(part, data[24:64])
    every = np.zeros(16 * 8, np.uint32)
    L.readU256DataFile_h(every.ctypes.data, p, 64, 16)          # every 4th element
    assert np.array_equal(every.reshape(16, 8), data.reshape(64, 8)[::4])
    same = np.zeros(64 * 8, np.uint32)
    L.readU256DataFile_h(same.ctypes.data, p, 64, 64)
    assert np.array_equal(same, data)
    w = data.reshape(64, 8)[:10]
    wp = str(tmp_path / "w.bin").encode()
    L.writeWitnessFile_h(np.ascontiguousarray(w).ctypes.data, wp, 10)
    assert np.array_equal(np.fromfile(wp.decode(), dtype="<u4"), pkfile.write_witness_bin(w))
    back = np.zeros((10, 8), np.uint32)
    L.readWitnessFile_h(back.ctypes.data, wp, 1, 10)
    assert np.array_equal(back, w)
    assert L.get_nprocs_h() >= 1


def test_isinf_matches_reference(golden):
    """ec_isinf / ec2_isinf with the reference's row addressing, for both moduli."""
    g = golden("dropin.npz")
    for ec2, fn in ((0, lib().ec_isinf), (1, lib().ec2_isinf)):
        pre = f"g{ec2 + 1}_"
        for tag, pidx in (("", 0), ("_p1", 1)):
            flat = np.ascontiguousarray(g[pre + "isinf_in" + tag])
            want = g[pre + "isinf" + tag]
            z = np.zeros(want.size, np.uint32)
            fn(z.ctypes.data, flat.ctypes.data, want.size, pidx)
            assert np.array_equal(z, want), (ec2, tag)


def test_range_and_add_match_reference(golden):
    g = golden("dropin.npz")
    L = lib()
    start = np.ascontiguousarray(g["range_start"]); mod = np.ascontiguousarray(g["range_mod"])
    out = np.zeros((12, 8), np.uint32)
    L.rangeu256_h(out.ctypes.data, 12, start.ctypes.data, 3, mod.ctypes.data)
    assert np.array_equal(out, g["range_3"])
    out = np.zeros((12, 8), np.uint32)
    L.rangeu256_h(out.ctypes.data, 12, start.ctypes.data, 7, None)
    assert np.array_equal(out, g["range_7_nomod"])
    a = np.array([0xffffffff] * 8, np.uint32); b = np.array([2] + [0] * 7, np.uint32)
    u = np.zeros(8, np.uint32)
    L.addu256_h(u.ctypes.data, a.ctypes.data, b.ctypes.data)
    assert list(u) == [1] + [0] * 7  # mod 2^256


def test_file_headers(tmp_path):
    """readU256PKFileHeader_h takes the nine leading words in order (its domainSize field gets
    the file's domainBits word, as the reference's does); readU256CircuitFileHeader_h nine
    uint64 words."""
    from cusnarks_b200._lib import lib as _l
    import ctypes as C

    class PkHdr(C.Structure):
        _fields_ = [(n, C.c_uint32) for n in ("nWords", "ftype", "protocol", "Rbitlen", "k_binformat",
                                              "k_ecformat", "nVars", "nPublic", "domainSize")]

    class CirHdr(C.Structure):
        _fields_ = [(n, C.c_ulonglong) for n in ("nWords", "nPubInputs", "nOutputs", "nVars", "nConstraints",
                                                 "cirformat", "R1CSA_nWords", "R1CSB_nWords", "R1CSC_nWords")]

    words = np.array([1000, 1, 1, 256, 1, 2, 20, 1, 5, 32] + [0] * 8, np.uint32)
    p = tmp_path / "pk.bin"
    words.tofile(p)
    h = PkHdr()
    _l().readU256PKFileHeader_h(C.byref(h), str(p).encode())
    assert [getattr(h, f) for f, _ in PkHdr._fields_] == list(words[:9])
    w64 = np.arange(10, 19, dtype=np.uint64)
    q = tmp_path / "c.bin"
    w64.tofile(q)
    c = CirHdr()
    _l().readU256CircuitFileHeader_h(C.byref(c), str(q).encode())
    assert [getattr(c, f) for f, _ in CirHdr._fields_] == list(w64)
