"""The benchmark circuit and its Groth16 proving key, built on the CPU.

TEST INFRASTRUCTURE ONLY.  bench.py's reference arm times the reference's own CPU prover
(oracle/_ref) and must not load the CUDA library, so it cannot use
cusnarks_b200.groth.SyntheticCircuit / setup_pk, which run their field and curve work
on the GPU.  This module builds the same circuit and key without a GPU:

* the draws (wires, coefficients, inputs, toxic waste) come from the same seeded
  streams through cusnarks_b200.groth.CircuitPlan / toxic_waste, which are numpy code
  and load no shared library;
* the arithmetic (Montgomery conversion, witness rows, Lagrange basis at t, wire
  polynomials, C and H scalars, fixed-base multiplications of the generators) runs in
  the oracle's C library (cs_oracle.c: or_r1cs_eval, or_lagrange_at, or_wire_eval,
  or_c_scalars, or_pow_scalars, or_fixed_base_mul), following Groth16 setup as the
  reference computes it (src/python/groth_setup.py:488-742).

Field and curve results are canonical, so the arrays equal the GPU builder's word for
word (tests/test_gpu_config_sizes.py compares them).
"""
from __future__ import annotations

import ctypes

import numpy as np

from .oracle import Oracle, _p, R, ints_to_limbs

MONT = 1 << 256


def _mont(x: int) -> np.ndarray:
    return ints_to_limbs([(x * MONT) % R])[0]


class CpuCircuit:
    """Attributes as cusnarks_b200.groth.SyntheticCircuit (w, polsA/B/C, a/b wires and
    Montgomery coefficients, sizes), computed on the host."""

    def __init__(self, o: Oracle, log_m: int, seed: int = 1, n_public: int = 1, n_inputs: int = 64):
        from cusnarks_b200.groth import CircuitPlan
        plan = CircuitPlan(log_m, seed, n_public, n_inputs)
        for k in ("log_m", "m", "n_public", "n_constraints", "n_inputs", "n_vars", "layers", "a_wire", "b_wire"):
            setattr(self, k, getattr(plan, k))
        nc = self.n_constraints
        coeff_m = o.to_mont(plan.coeff, 1).reshape(nc, 6, 8)
        self.a_coeff = np.ascontiguousarray(coeff_m[:, :3])
        self.b_coeff = np.ascontiguousarray(coeff_m[:, 3:])
        w = np.ascontiguousarray(plan.initial_witness())
        aw = np.ascontiguousarray(self.a_wire.reshape(-1))
        bw = np.ascontiguousarray(self.b_wire.reshape(-1))
        o.lib.or_r1cs_eval(_p(w), ctypes.c_uint64(self.n_inputs), ctypes.c_uint64(nc), 3, _p(aw),
                           _p(self.a_coeff.reshape(-1)), _p(bw), _p(self.b_coeff.reshape(-1)))
        self.w = w
        self.polsA, self.polsB, self.polsC = plan.matrices(self.a_coeff, self.b_coeff)

    @property
    def public_inputs(self) -> np.ndarray:
        return self.w[1:self.n_public + 1]


def fixed_base_mul(o: Oracle, scal: np.ndarray, ec2: bool = False) -> np.ndarray:
    """k_i * G for normal-form scalars k_i and the G1 (or G2) generator; affine Montgomery."""
    from .oracle import G1_GEN, G2_GEN, to_mont_int
    if ec2:
        g = ints_to_limbs([to_mont_int(c, 0) for xy in G2_GEN for c in xy]).reshape(-1)
    else:
        g = ints_to_limbs([to_mont_int(c, 0) for c in G1_GEN]).reshape(-1)
    scal = np.ascontiguousarray(scal, dtype=np.uint32).reshape(-1, 8)
    out = np.zeros((scal.shape[0], 32 if ec2 else 16), dtype=np.uint32)
    o.lib.or_fixed_base_mul(_p(out), _p(scal), ctypes.c_uint64(scal.shape[0]), _p(np.ascontiguousarray(g)),
                            1 if ec2 else 0)
    return out


def cpu_setup_pk(o: Oracle, circ: CpuCircuit, seed: int = 7) -> dict:
    """The proving key cusnarks_b200.groth.setup_pk makes for the same circuit and seed, in
    the host layout cusnarks_b200.groth.pk_to_host returns."""
    from cusnarks_b200.groth import toxic_waste
    t, alpha, beta, gamma, delta = toxic_waste(seed)
    m, nv, npub = circ.m, circ.n_vars, circ.n_public
    tm = _mont(t)
    Lc = np.zeros((m, 8), dtype=np.uint32)
    o.lib.or_lagrange_at(_p(Lc), circ.log_m, _p(tm))
    uvw = []
    for pol in (circ.polsA, circ.polsB, circ.polsC):
        out = np.zeros((nv, 8), dtype=np.uint32)
        o.lib.or_wire_eval(_p(out), _p(np.ascontiguousarray(pol)), _p(Lc), m)
        uvw.append(out)
    u, v, w = uvw
    nu, nvv = o.from_mont(u, 1), o.from_mont(v, 1)
    A = fixed_base_mul(o, nu)
    B1 = fixed_base_mul(o, nvv)
    B2 = fixed_base_mul(o, nvv, ec2=True)

    def c_scalars(k: int, n: int) -> np.ndarray:
        out = np.zeros((n, 8), dtype=np.uint32)
        o.lib.or_c_scalars(_p(out), _p(u), _p(v), _p(w), _p(_mont(alpha)), _p(_mont(beta)),
                           _p(_mont(pow(k, -1, R))), ctypes.c_uint64(n))
        return out

    C = fixed_base_mul(o, c_scalars(delta, nv))
    IC = fixed_base_mul(o, c_scalars(gamma, npub + 1))
    zt = (pow(t, m, R) - 1) % R
    hs = np.zeros((m - 1, 8), dtype=np.uint32)
    o.lib.or_pow_scalars(_p(hs), _p(tm), _p(_mont(zt * pow(delta, -1, R) % R)), ctypes.c_uint64(m - 1))
    H = fixed_base_mul(o, hs)
    alpha1, beta1, delta1 = (fixed_base_mul(o, ints_to_limbs([x])) for x in (alpha, beta, delta))
    beta2, gamma2, delta2 = (fixed_base_mul(o, ints_to_limbs([x]), ec2=True) for x in (beta, gamma, delta))
    return {
        "n_vars": nv, "n_public": npub, "domain_size": m,
        "polsA": circ.polsA, "polsB": circ.polsB,
        "A": np.concatenate([A, alpha1, delta1]), "B1": np.concatenate([B1, beta1, delta1]),
        "B2": np.concatenate([B2, beta2, delta2]), "C": C, "hExps": H, "delta_1": delta1,
        "vk": {"alpha_1": alpha1.reshape(16), "beta_2": beta2.reshape(32), "gamma_2": gamma2.reshape(32),
               "delta_2": delta2.reshape(32), "IC": IC.reshape(-1, 16)},
    }
