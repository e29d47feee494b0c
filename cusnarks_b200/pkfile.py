"""Proving-key and witness files in the reference's binary formats.

Proving key `.bin` (README.md "Proving Key .bin"; writer src/python/pysnarks_utils.py:619
pkvars_to_bin, reader :544 pkbin_get), little-endian uint32 words:

    [0] nWords  [1] ftype (1 = proving key)  [2] protocol (1 = Groth16)  [3] Rbitlen (256)
    [4] k_binformat (1 Montgomery, 0 normal)  [5] k_ecformat (2 affine)  [6] nVars  [7] nPublic
    [8] domainBits  [9] domainSize  [10..17] field r  [18..25] group q
    [26..39] word counts (uint64 low word first) of polsA, polsB, A, B1, B2, C, hExps
    polsA, polsB (mpoly layout), alfa_1, beta_1, delta_1 (G1), beta_2, delta_2 (G2),
    A, B1, B2, C, hExps (affine points; with the extension, A/B1/B2 carry alfa_1/delta_1,
    beta_1/delta_1, beta_2/delta_2 after their nVars points).

Witness `.bin` (src/cuda/file_utils.cpp:550 readWitnessFile_h, fmt 1): a 4-word header
(uint64 count, word size, reserved) then the values; `.dat` (fmt 0): values from byte 32.
`.json` / `.txt`: decimal integers.  Witness values are normal-form Fr elements.

`read_pk_bin` returns the dictionary `groth.Prover` takes (host arrays, Montgomery form).
"""
from __future__ import annotations

import json
import os

import numpy as np

HDR_WORDS = 10
FMT_EXT, FMT_MONT = 0, 1
EC_T_AFFINE = 2
SNARKSFILE_T_PK = 1
PROTOCOL_T_GROTH = 1
R = 21888242871839275222246405745257275088548364400416034343698204186575808495617
Q = 21888242871839275222246405745257275088696311157297823662689037894645226208583
_NAMES = ("polsA", "polsB", "A", "B1", "B2", "C", "hExps")


def _limbs(x: int) -> np.ndarray:
    return np.array([(x >> (32 * i)) & 0xffffffff for i in range(8)], dtype=np.uint32)


def _u64(w: np.ndarray, i: int) -> int:
    return int(w[i]) | (int(w[i + 1]) << 32)


def _dw(x: int) -> np.ndarray:
    return np.array([x & 0xffffffff, x >> 32], dtype=np.uint32)


def read_pk_bin(src, ctx=None) -> dict:
    """src: path or uint32 array.  Keys: n_vars, n_public, domain_size, polsA, polsB, A, B1 (nVars+2
    G1 rows of 16 words), B2 (nVars+2 G2 rows of 32), C (nVars rows), hExps (domain_size-1 rows),
    delta_1, and the single points alfa_1, beta_1, beta_2, delta_2.  A file in normal form
    (k_binformat 0) is converted to Montgomery form on the GPU (ctx required)."""
    w = np.fromfile(src, dtype="<u4") if isinstance(src, (str, os.PathLike)) else np.asarray(src, dtype=np.uint32)
    if w.size < HDR_WORDS + 16 + 14:
        raise ValueError("proving key file too short")
    if int(w[1]) != SNARKSFILE_T_PK or int(w[2]) != PROTOCOL_T_GROTH:
        raise ValueError(f"not a Groth16 proving key (ftype {int(w[1])}, protocol {int(w[2])})")
    if int(w[5]) != EC_T_AFFINE:
        raise ValueError(f"unsupported point format {int(w[5])} (affine expected)")
    binfmt = int(w[4])
    nv, npub, m = int(w[6]), int(w[7]), int(w[9])
    cnt = {k: _u64(w, HDR_WORDS + 16 + 2 * i) for i, k in enumerate(_NAMES)}
    o = HDR_WORDS + 16 + 14
    polsA = w[o:o + cnt["polsA"]]
    o += cnt["polsA"]
    polsB = w[o:o + cnt["polsB"]]
    o += cnt["polsB"]
    alfa_1, beta_1, delta_1 = w[o:o + 16], w[o + 16:o + 32], w[o + 32:o + 48]
    beta_2, delta_2 = w[o + 48:o + 80], w[o + 80:o + 112]
    o += 112
    sec = {}
    for k in ("A", "B1", "B2", "C", "hExps"):
        sec[k] = w[o:o + cnt[k]]
        o += cnt[k]
    if o > w.size:
        raise ValueError("proving key file truncated")

    def pts(a, pw, n):
        a = np.asarray(a).reshape(-1, pw)
        if a.shape[0] < n:
            raise ValueError("proving key section shorter than its point count")
        return a[:n]

    def ext(a, pw, tail):
        a = np.asarray(a).reshape(-1, pw)
        if a.shape[0] >= nv + 2:
            return a[:nv + 2].copy()
        return np.concatenate([pts(a, pw, nv)] + [np.asarray(t).reshape(1, pw) for t in tail])

    pk = {
        "n_vars": nv, "n_public": npub, "domain_size": m,
        "polsA": np.ascontiguousarray(polsA), "polsB": np.ascontiguousarray(polsB),
        "A": ext(sec["A"], 16, (alfa_1, delta_1)),
        "B1": ext(sec["B1"], 16, (beta_1, delta_1)),
        "B2": ext(sec["B2"], 32, (beta_2, delta_2)),
        "C": pts(sec["C"], 16, nv).copy(),
        "hExps": pts(sec["hExps"], 16, m - 1).copy(),
        "delta_1": delta_1.reshape(1, 16).copy(),
        "alfa_1": alfa_1.copy(), "beta_1": beta_1.copy(), "beta_2": beta_2.copy(), "delta_2": delta_2.copy(),
    }
    if binfmt == FMT_EXT:
        _to_montgomery(pk, ctx)
    elif binfmt != FMT_MONT:
        raise ValueError(f"unknown field format {binfmt}")
    return pk


def _to_montgomery(pk: dict, ctx):
    """Normal-form key -> Montgomery form with the library's field kernel (coordinates mod q,
    mpoly coefficients mod r)."""
    if ctx is None:
        raise ValueError("a normal-form proving key needs a Context for the conversion")
    import torch

    def conv(a: np.ndarray, pidx: int) -> np.ndarray:
        flat = np.ascontiguousarray(a, dtype=np.uint32).reshape(-1, 8)
        d = torch.from_numpy(flat.view(np.int32)).cuda(ctx.device)
        torch.cuda.synchronize()
        ctx.field_op_device("to_mont", pidx, d.data_ptr(), 0, d.data_ptr(), flat.shape[0])
        ctx.sync()
        return d.cpu().numpy().view(np.uint32).reshape(a.shape)

    for k in ("A", "B1", "B2", "C", "hExps", "delta_1", "alfa_1", "beta_1", "beta_2", "delta_2"):
        pk[k] = conv(pk[k], 0)
    for k in ("polsA", "polsB"):
        p = pk[k].copy()
        nw = int(p[0])
        counts = p[1:1 + nw].astype(np.int64)
        base = 1 + nw
        for c in counts:
            vals = p[base + c:base + c + 8 * c].reshape(-1, 8)
            if c:
                p[base + c:base + c + 8 * c] = conv(vals, 1).reshape(-1)
            base += 9 * int(c)
        pk[k] = p


def write_pk_bin(pk: dict, path=None) -> np.ndarray:
    """Writes a Montgomery-form, affine, extended proving key in the layout of the reference's
    pkvars_to_bin(FMT_MONT, EC_T_AFFINE, pk, ext=True).  pk: read_pk_bin's keys (A/B1/B2 with
    nVars+2 rows).  Returns the words; writes them to path when given."""
    nv, npub, m = int(pk["n_vars"]), int(pk["n_public"]), int(pk["domain_size"])
    bits = m.bit_length() - 1
    A = np.asarray(pk["A"], dtype=np.uint32).reshape(-1, 16)
    B1 = np.asarray(pk["B1"], dtype=np.uint32).reshape(-1, 16)
    B2 = np.asarray(pk["B2"], dtype=np.uint32).reshape(-1, 32)
    C = np.asarray(pk["C"], dtype=np.uint32).reshape(-1)
    H = np.asarray(pk["hExps"], dtype=np.uint32).reshape(-1)
    d1 = np.asarray(pk["delta_1"], dtype=np.uint32).reshape(-1)
    a1 = np.asarray(pk.get("alfa_1", A[nv]), dtype=np.uint32).reshape(-1)
    b1 = np.asarray(pk.get("beta_1", B1[nv]), dtype=np.uint32).reshape(-1)
    b2 = np.asarray(pk.get("beta_2", B2[nv]), dtype=np.uint32).reshape(-1)
    d2 = np.asarray(pk.get("delta_2", B2[nv + 1]), dtype=np.uint32).reshape(-1)
    pA = np.asarray(pk["polsA"], dtype=np.uint32).reshape(-1)
    pB = np.asarray(pk["polsB"], dtype=np.uint32).reshape(-1)
    # extension sizes as the reference writer computes them
    pA_n = max(pA.size, m * 8)
    pB_n = max(pB.size, m * 8)
    A_n, B1_n, B2_n = nv * 16 + 32, nv * 16 + 32, nv * 32 + 64
    C_n, H_n = C.size, H.size + 96
    h_ext = np.zeros(H.size, dtype=np.uint32)
    h_ext[48:64] = d1[:16] if H.size >= 64 else 0
    hdr = np.array([0, SNARKSFILE_T_PK, PROTOCOL_T_GROTH, 256, FMT_MONT, EC_T_AFFINE, nv, npub, bits, m],
                   dtype=np.uint32)
    words = np.concatenate([
        hdr, _limbs(R), _limbs(Q),
        _dw(pA_n), _dw(pB_n), _dw(A_n), _dw(B1_n), _dw(B2_n), _dw(C_n), _dw(H_n),
        pA, np.zeros(pA_n - pA.size, np.uint32), pB, np.zeros(pB_n - pB.size, np.uint32),
        a1, b1, d1, b2, d2,
        A[:nv].reshape(-1), a1, d1,
        B1[:nv].reshape(-1), b1, d1,
        B2[:nv].reshape(-1), b2, d2,
        C, H, h_ext])
    words[0] = words.size
    if path is not None:
        words.astype("<u4").tofile(path)
    return words


def read_witness(path, n_vars: int) -> np.ndarray:
    """Witness file -> (n_vars, 8) normal-form limbs (.bin, .dat, .json, .txt, as the reference
    prover's read_witness_data, groth_prover.py:963-1004)."""
    p = str(path)
    if p.endswith(".bin") or p.endswith(".dat"):
        w = np.fromfile(p, dtype="<u4")
        start = 4 if p.endswith(".bin") else 8
        vals = w[start:start + 8 * n_vars]
        if vals.size < 8 * n_vars:
            raise ValueError("witness file shorter than n_vars values")
        return vals.reshape(n_vars, 8).copy()
    if p.endswith(".json"):
        with open(p) as f:
            ints = [int(x) for x in json.load(f)]
    elif p.endswith(".txt"):
        with open(p) as f:
            ints = [int(line) for line in f if line.strip()]
    else:
        raise ValueError(f"unknown witness file type: {p}")
    if len(ints) < n_vars:
        raise ValueError("witness file shorter than n_vars values")
    return np.stack([_limbs(x % (1 << 256)) for x in ints[:n_vars]])


def write_witness_bin(w: np.ndarray, path=None) -> np.ndarray:
    """The reference's writeWitnessFile_h layout (file_utils.cpp:583): uint64 count, word size 8,
    reserved 0, then the values."""
    w = np.ascontiguousarray(w, dtype=np.uint32).reshape(-1, 8)
    words = np.concatenate([_dw(w.shape[0]), np.array([8, 0], np.uint32), w.reshape(-1)])
    if path is not None:
        words.astype("<u4").tofile(path)
    return words
