"""Shared helpers for the GPU parity tests: seeded inputs and a session context."""
import numpy as np
import pytest

from oracle.oracle import (G1_GEN, G2_GEN, ints_to_limbs, random_field, to_mont_int)


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def g1_generator_mont():
    return np.concatenate([ints_to_limbs([to_mont_int(c, 0)]) for c in G1_GEN]).reshape(16)


def g2_generator_mont():
    return np.concatenate([ints_to_limbs([to_mont_int(c, 0) for c in xy]) for xy in G2_GEN]).reshape(32)


def random_points(oracle, rng, n, ec2=False):
    """n points k_i * G with k_i uniform in Fr (seeded), affine Montgomery."""
    g = g2_generator_mont() if ec2 else g1_generator_mont()
    k = random_field(rng, n, 1)
    return oracle.scmul(k, g.reshape(1, -1), 1 if ec2 else 0)
