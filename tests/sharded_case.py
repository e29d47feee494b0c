"""Seeded MSM inputs shared by the sharded-MSM tests (points k*G made by the oracle)."""
import numpy as np


def case(n: int, ec2: bool):
    from oracle.oracle import Oracle, random_field, G1_GEN, G2_GEN, ints_to_limbs, to_mont_int
    o = Oracle()
    rng = np.random.Generator(np.random.PCG64(4242 + n + 1000 * int(ec2)))
    if ec2:
        g = np.concatenate([ints_to_limbs([to_mont_int(c, 0) for c in xy]) for xy in G2_GEN]).reshape(1, 32)
    else:
        g = np.concatenate([ints_to_limbs([to_mont_int(c, 0)]) for c in G1_GEN]).reshape(1, 16)
    pts = np.asarray(o.scmul(random_field(rng, n, 1), g, int(ec2))).reshape(n, -1).astype(np.uint32)
    scl = random_field(rng, n, 1)
    return np.ascontiguousarray(scl), np.ascontiguousarray(pts)
