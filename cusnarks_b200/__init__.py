"""cusnarks_b200 -- Blackwell (sm_100a) Groth16/BN128 prover hot path.

The compute lives in ``libcusnarks_b200.so`` (CUDA kernels behind the C ABI declared in
include/cusnarks_b200.h).  ``pycusnarks`` mirrors the reference's Cython functions on this
path; ``Context`` exposes the context/device-pointer API.
"""
from ._lib import CsError, lib, exported_symbols  # noqa: F401
from .context import Context  # noqa: F401

__all__ = ["CsError", "lib", "exported_symbols", "Context"]
