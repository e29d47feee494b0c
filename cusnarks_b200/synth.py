"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public dataset is involved in the reference's benchmarks; these generators produce the
inputs its configurations describe: field elements uniform in [0, p) from a seeded
numpy PCG64 stream (rejection sampling on 8 x 32-bit limbs), and curve points k_i * G with
seeded k_i, computed on the GPU by the library's batched scalar multiplication.
"""
from __future__ import annotations

import numpy as np

Q = 21888242871839275222246405745257275088696311157297823662689037894645226208583
R = 21888242871839275222246405745257275088548364400416034343698204186575808495617
MONT = 1 << 256

G1_GEN = (1, 2)
G2_GEN = (
    (10857046999023057135944570762232829481370756359578518086990519993285655852781,
     11559732032986387107991004021392285783925812861821192530917403151452391805634),
    (8495653923123431417604973247489272438418190587263600148770280649306958101930,
     4082367875863433681332203403145435568316851327593401208105741076214120093531),
)


def to_limbs(x: int) -> np.ndarray:
    return np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(8)], dtype=np.uint32)


def from_limbs(a) -> int:
    a = np.asarray(a, dtype=np.uint64).reshape(-1)
    v = 0
    for i in range(7, -1, -1):
        v = (v << 32) | int(a[i])
    return v


def mont(x: int, p: int = Q) -> np.ndarray:
    return to_limbs((x * MONT) % p)


def g1_generator() -> np.ndarray:
    return np.concatenate([mont(G1_GEN[0]), mont(G1_GEN[1])])


def g2_generator() -> np.ndarray:
    (x0, x1), (y0, y1) = G2_GEN
    return np.concatenate([mont(x0), mont(x1), mont(y0), mont(y1)])


def random_field(rng: np.random.Generator, n: int, p: int = R) -> np.ndarray:
    """(n, 8) uint32, uniform in [0, p) by rejection on the top limb then exact compare.
    p is the modulus itself (R or Q), at least 2^224 so a candidate passes with probability
    at least 1/2 (a field index such as 1 would reject every candidate but zero)."""
    if p < (1 << 224) or p >= (1 << 256):
        raise ValueError("random_field: p must be a modulus in [2^224, 2^256)")
    top = p >> 224
    out = np.empty((n, 8), dtype=np.uint32)
    filled = 0
    while filled < n:
        k = max(64, int((n - filled) * 1.02) + 64)
        cand = rng.integers(0, 1 << 32, size=(k, 8), dtype=np.uint64).astype(np.uint32)
        cand[:, 7] %= np.uint32(top + 1)
        ok = cand[:, 7] < top
        for i in np.nonzero(cand[:, 7] == top)[0]:
            ok[i] = from_limbs(cand[i]) < p
        good = cand[ok]
        take = min(len(good), n - filled)
        out[filled:filled + take] = good[:take]
        filled += take
    return out
