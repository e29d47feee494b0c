"""Drop-in mirror of the reference's ``pycusnarks`` functions on the prover hot path.

Same names, argument order and return shapes as the reference Cython wrappers in
src/cython/_cusnarks_kernel.pyx, but every call goes through this repository's C ABI
(include/cusnarks_b200.h) and runs on the GPU.  Where the reference exits the process on
an error, these raise ``CsError``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import lib, check, JacaddReduced, CsError

NWORDS_256BIT = 8
ECP_JAC_INDIMS = 2
ECP_JAC_OUTDIMS = 3
ECP2_JAC_INDIMS = 4
ECP2_JAC_OUTDIMS = 6
MOD_GROUP = 0
MOD_FIELD = 1


def ec_jacreduce_h(inscl, intbl, fname: bytes, offset: int, total_words: int, order: int,
                   ec2: int, pidx: int, to_aff: int, add_in: int, strip_last: int,
                   pippen_conf: int) -> np.ndarray:
    """Multi-exponentiation (reference _cusnarks_kernel.pyx:992 -> ec_jacreduce_server_h).

    inscl: flat uint32 scalars (n x 8, normal form); intbl: flat affine Montgomery points.
    Returns the affine result reshaped to (-1, 8): X, Y (G1) or X.c0, X.c1, Y.c0, Y.c1
    (G2), padded with zero rows to the reference's output length when strip_last == 0.
    """
    outdims = ECP_JAC_INDIMS if strip_last else ECP_JAC_OUTDIMS
    if ec2:
        outdims = ECP2_JAC_INDIMS if strip_last else ECP2_JAC_OUTDIMS
    if fname:
        raise CsError(4, "precomputed EC table files are not supported by the GPU path")
    scl = np.ascontiguousarray(inscl, dtype=np.uint32).reshape(-1)
    pts = np.ascontiguousarray(intbl, dtype=np.uint32).reshape(-1)
    n = scl.shape[0] // NWORDS_256BIT
    indims = ECP2_JAC_INDIMS if ec2 else ECP_JAC_INDIMS
    if pts.shape[0] < n * indims * NWORDS_256BIT:
        raise ValueError("point table shorter than the scalar vector")
    outv = np.zeros(outdims * NWORDS_256BIT, dtype=np.uint32)
    args = JacaddReduced()
    args.out_ep = outv.ctypes.data
    args.scl = scl.ctypes.data
    args.x = pts.ctypes.data
    args.n = n
    args.ec2 = 1 if ec2 else 0
    args.pidx = pidx
    args.order = order
    args.pippen = pippen_conf
    args.offset = offset
    args.total_words = total_words
    args.filename = None
    L = lib()
    L.ec_jacreduce_server_h(ctypes.byref(args))
    check(L.cs_last_status())
    return np.reshape(outv, (-1, NWORDS_256BIT))
