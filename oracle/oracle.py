"""CPU checkers for the Groth16/BN128 prover hot path.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline leg import this module.  The product library (``cusnarks_b200``) never imports,
links or calls anything under ``oracle/``.

Two checkers live behind this module:

* ``Oracle``   -- ``liboracle.so``, this repository's C restatement of the reference
  algorithms (``cs_oracle.c``), with the reference file:line each function follows.
* ``RefLib``   -- ``_ref/libcusnarks_ref.so``, the reference's own host C++ compiled from
  its sources by ``oracle/Makefile`` (``make ref``).  It exists only where the reference
  tree was present at build time; callers must handle ``RefLib.available() == False``.

Arrays are numpy uint32 with 8 little-endian limbs per field element, the layout the
reference uses everywhere (src/cuda/types.h: NWORDS_256BIT).
"""
from __future__ import annotations

import ctypes
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

Q = 21888242871839275222246405745257275088696311157297823662689037894645226208583
R = 21888242871839275222246405745257275088548364400416034343698204186575808495617
MOD = {0: Q, 1: R}
MONT_R = 1 << 256

G1_GEN = (1, 2)
G2_GEN = (
    (10857046999023057135944570762232829481370756359578518086990519993285655852781,
     11559732032986387107991004021392285783925812861821192530917403151452391805634),
    (8495653923123431417604973247489272438418190587263600148770280649306958101930,
     4082367875863433681332203403145435568316851327593401208105741076214120093531),
)

_u32p = ctypes.POINTER(ctypes.c_uint32)


def _p(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_u32p)


# ----------------------------------------------------------------- conversions ------
def int_to_limbs(x: int) -> np.ndarray:
    return np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(8)], dtype=np.uint32)


def ints_to_limbs(xs) -> np.ndarray:
    out = np.zeros((len(xs), 8), dtype=np.uint32)
    for k, x in enumerate(xs):
        for i in range(8):
            out[k, i] = (x >> (32 * i)) & 0xFFFFFFFF
    return out


def limbs_to_int(a) -> int:
    a = np.asarray(a, dtype=np.uint64).reshape(-1)
    v = 0
    for i in range(7, -1, -1):
        v = (v << 32) | int(a[i])
    return v


def limbs_to_ints(a) -> list:
    a = np.asarray(a, dtype=np.uint32).reshape(-1, 8)
    return [limbs_to_int(row) for row in a]


def to_mont_int(x: int, pidx: int) -> int:
    return (x * MONT_R) % MOD[pidx]


def from_mont_int(x: int, pidx: int) -> int:
    return (x * pow(MONT_R, -1, MOD[pidx])) % MOD[pidx]


# ----------------------------------------------------------- seeded generators -----
def random_field(rng: np.random.Generator, n: int, pidx: int = 1) -> np.ndarray:
    """n uniform elements of [0, p) as (n, 8) uint32, rejection sampled on 8x32 limbs."""
    p = MOD[pidx]
    top = p >> 224
    out = np.empty((n, 8), dtype=np.uint32)
    filled = 0
    while filled < n:
        k = max(16, int((n - filled) * 1.3))
        cand = rng.integers(0, 1 << 32, size=(k, 8), dtype=np.uint64).astype(np.uint32)
        cand[:, 7] = cand[:, 7] % np.uint32(top + 1)
        ok = cand[:, 7] < top
        # rows whose top limb equals top(p) need an exact comparison
        eq = np.nonzero(cand[:, 7] == top)[0]
        for i in eq:
            ok[i] = limbs_to_int(cand[i]) < p
        good = cand[ok]
        take = min(len(good), n - filled)
        out[filled:filled + take] = good[:take]
        filled += take
    return out


# ------------------------------------------------------------------- restatement ----
class Oracle:
    """ctypes front-end to liboracle.so (cs_oracle.c)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle)")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.or_ntt.argtypes = [_u32p, _u32p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64,
                             ctypes.c_int32, ctypes.c_uint32]
        L.or_intt.argtypes = [_u32p, _u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                              ctypes.c_uint32]
        L.or_interpolandmul.argtypes = [_u32p, _u32p, _u32p, _u32p, ctypes.c_uint32, ctypes.c_uint64]
        L.or_ec_isoncurve_aff.restype = ctypes.c_uint32

    # field ---------------------------------------------------------------------
    def montmult(self, a, b, pidx):
        a = np.ascontiguousarray(a, dtype=np.uint32).reshape(-1, 8)
        b = np.ascontiguousarray(b, dtype=np.uint32).reshape(-1, 8)
        z = np.zeros_like(a)
        for i in range(a.shape[0]):
            self.lib.or_montmult(_p(z[i]), _p(a[i]), _p(b[i]), pidx)
        return z

    def to_mont(self, a, pidx):
        a = np.ascontiguousarray(a, dtype=np.uint32).reshape(-1, 8)
        z = np.zeros_like(a)
        self.lib.or_to_mont(_p(z), _p(a), a.shape[0], pidx)
        return z

    def from_mont(self, a, pidx):
        a = np.ascontiguousarray(a, dtype=np.uint32).reshape(-1, 8)
        z = np.zeros_like(a)
        self.lib.or_from_mont(_p(z), _p(a), a.shape[0], pidx)
        return z

    def const(self, pidx):
        one = np.zeros(8, np.uint32)
        r2 = np.zeros(8, np.uint32)
        self.lib.or_get_const(_p(one), _p(r2), pidx)
        return one, r2

    # curve ---------------------------------------------------------------------
    def scmul(self, scl, pts_aff, ec2=0):
        """per-point k_i * P_i, affine Montgomery out."""
        scl = np.ascontiguousarray(scl, dtype=np.uint32).reshape(-1, 8)
        w = 32 if ec2 else 16
        pts = np.ascontiguousarray(pts_aff, dtype=np.uint32).reshape(-1, w)
        if pts.shape[0] == 1 and scl.shape[0] > 1:
            pts = np.ascontiguousarray(np.repeat(pts, scl.shape[0], axis=0))
        out = np.zeros((scl.shape[0], w), dtype=np.uint32)
        self.lib.or_ec_scmul(_p(out), _p(scl), _p(pts), scl.shape[0], ec2)
        return out

    def isoncurve(self, pt_aff, ec2=0):
        pt = np.ascontiguousarray(pt_aff, dtype=np.uint32).reshape(-1)
        return bool(self.lib.or_ec_isoncurve_aff(_p(pt), ec2))

    def jac2aff(self, jac, ec2=0):
        w = 48 if ec2 else 24
        jac = np.ascontiguousarray(jac, dtype=np.uint32).reshape(-1, w)
        out = np.zeros((jac.shape[0], w * 2 // 3), dtype=np.uint32)
        self.lib.or_ec_jac2aff(_p(out), _p(jac), jac.shape[0], ec2)
        return out

    def msm(self, scl, pts_aff, ec2=0, order=6, nthreads=0):
        scl = np.ascontiguousarray(scl, dtype=np.uint32).reshape(-1, 8)
        w = 32 if ec2 else 16
        pts = np.ascontiguousarray(pts_aff, dtype=np.uint32).reshape(-1, w)
        assert pts.shape[0] == scl.shape[0]
        out = np.zeros(w, dtype=np.uint32)
        self.lib.or_msm(_p(out), _p(scl), _p(pts), scl.shape[0], ec2, order, nthreads)
        return out

    # transforms ----------------------------------------------------------------
    def find_roots(self, levels):
        out = np.zeros((1 << levels, 8), dtype=np.uint32)
        self.lib.or_find_roots(_p(out), levels)
        return out

    def root_powers(self, proot, n):
        proot = np.ascontiguousarray(proot, dtype=np.uint32).reshape(8)
        out = np.zeros((n, 8), dtype=np.uint32)
        self.lib.or_root_powers(_p(out), _p(proot), ctypes.c_uint64(n))
        return out

    def ntt(self, A, roots, levels, astride=1, rstride=1, direction=1, pidx=1):
        A = np.array(A, dtype=np.uint32, copy=True).reshape(-1, 8)
        roots = np.ascontiguousarray(roots, dtype=np.uint32)
        self.lib.or_ntt(_p(A), _p(roots), levels, astride, rstride, direction, pidx)
        return A

    def intt(self, A, roots, levels, rstride=1, fmat=1, pidx=1):
        A = np.array(A, dtype=np.uint32, copy=True).reshape(-1, 8)
        roots = np.ascontiguousarray(roots, dtype=np.uint32)
        self.lib.or_intt(_p(A), _p(roots), fmat, levels, rstride, pidx)
        return A

    def interpolandmul(self, A, B, roots, levels, rstride=2):
        A = np.ascontiguousarray(A, dtype=np.uint32).reshape(-1, 8)
        B = np.ascontiguousarray(B, dtype=np.uint32).reshape(-1, 8)
        roots = np.ascontiguousarray(roots, dtype=np.uint32)
        M = np.zeros((2 << levels, 8), dtype=np.uint32)
        self.lib.or_interpolandmul(_p(M), _p(A), _p(B), _p(roots), levels, rstride)
        return M

    def hstep_coset(self, A, B, C, levels):
        A = np.ascontiguousarray(A, dtype=np.uint32).reshape(-1, 8)
        B = np.ascontiguousarray(B, dtype=np.uint32).reshape(-1, 8)
        C = np.ascontiguousarray(C, dtype=np.uint32).reshape(-1, 8)
        H = np.zeros((1 << levels, 8), dtype=np.uint32)
        self.lib.or_hstep_coset(_p(H), _p(A), _p(B), _p(C), levels)
        return H

    def mpoly_eval(self, scalar, pin, ncoeff, start_idx, last_idx, pidx=1):
        scalar = np.ascontiguousarray(scalar, dtype=np.uint32).reshape(-1)
        pin = np.ascontiguousarray(pin, dtype=np.uint32).reshape(-1)
        out = np.zeros((ncoeff, 8), dtype=np.uint32)
        self.lib.or_mpoly_eval(_p(out), _p(scalar), _p(pin), start_idx, last_idx, pidx)
        return out


# ---------------------------------------------------------- reference library ------
class _JacaddReduced(ctypes.Structure):
    """jacadd_reduced_t, src/cuda/types.h:548-567."""
    _fields_ = [("out_ep", ctypes.c_void_p), ("scl", ctypes.c_void_p), ("x", ctypes.c_void_p),
                ("n", ctypes.c_uint32), ("ec2", ctypes.c_uint32), ("compute_table", ctypes.c_uint32),
                ("ec_table", ctypes.c_void_p), ("pidx", ctypes.c_uint32),
                ("max_threads", ctypes.c_uint32), ("start_idx", ctypes.c_uint32),
                ("last_idx", ctypes.c_uint32), ("thread_id", ctypes.c_uint32),
                ("pippen", ctypes.c_uint32), ("offset", ctypes.c_uint64),
                ("total_words", ctypes.c_uint64), ("order", ctypes.c_uint32),
                ("filename", ctypes.c_char_p)]


class _InterpolAndMul(ctypes.Structure):
    """ntt_interpolandmul_t, src/cuda/types.h:530-546."""
    _fields_ = [("A", ctypes.c_void_p), ("B", ctypes.c_void_p), ("roots", ctypes.c_void_p),
                ("Nrows", ctypes.c_uint32), ("Ncols", ctypes.c_uint32), ("mNrows", ctypes.c_uint32),
                ("mNcols", ctypes.c_uint32), ("nroots", ctypes.c_uint32), ("rstride", ctypes.c_uint32),
                ("pidx", ctypes.c_uint32), ("max_threads", ctypes.c_uint32),
                ("start_idx", ctypes.c_uint32), ("last_idx", ctypes.c_uint32),
                ("thread_id", ctypes.c_uint32)]


class _MpolyEval(ctypes.Structure):
    """mpoly_eval_t, src/cuda/types.h:516-528."""
    _fields_ = [("pout", ctypes.c_void_p), ("scalar", ctypes.c_void_p), ("pin", ctypes.c_void_p),
                ("reduce_coeff", ctypes.c_uint32), ("start_idx", ctypes.c_uint32),
                ("last_idx", ctypes.c_uint32), ("max_threads", ctypes.c_uint32),
                ("thread_id", ctypes.c_uint32), ("pidx", ctypes.c_uint32)]


class RefLib:
    """The reference's own CPU implementation (oracle/_ref/libcusnarks_ref.so).

    Its entry points carry C++ linkage, so they are bound by their mangled names.  The
    library's global scratch is set up once with the calls init_h() makes
    (src/cuda/init.cpp:44), with a 2^22-entry NTT buffer so H steps up to m = 2^21 fit,
    without init_h's cwd-relative config file lookup.
    """

    PATH = os.path.join(HERE, "_ref", "libcusnarks_ref.so")
    _inst = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.PATH)

    @classmethod
    def get(cls) -> "RefLib":
        if cls._inst is None:
            cls._inst = RefLib()
        return cls._inst

    def __init__(self):
        self.lib = ctypes.CDLL(self.PATH)
        L = self.lib
        L._Z12utils_init_hv()
        L._Z9ec_init_hv()
        L._Z10ntt_init_hj(ctypes.c_uint32(1 << 22))
        self._msm = L._Z21ec_jacreduce_server_hP16jacadd_reduced_t
        self._ntt = L._Z5ntt_hPjPKjjyyij
        self._ntt.argtypes = [_u32p, _u32p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64,
                              ctypes.c_int32, ctypes.c_uint32]
        self._intt = L._Z6intt_hPjPKjjjyj
        self._intt.argtypes = [_u32p, _u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                               ctypes.c_uint32]
        self._interp = L._Z27ntt_interpolandmul_server_hP20ntt_interpolandmul_t
        self._interp.restype = ctypes.POINTER(ctypes.c_uint32)
        self._mmul = L._Z10get_Mmul_hv
        self._mmul.restype = ctypes.POINTER(ctypes.c_uint32)
        self._nttp = L._Z14ntt_parallel_hPjPKjjjyi10fft_mode_tj
        self._nttp.argtypes = [_u32p, _u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                               ctypes.c_int32, ctypes.c_int, ctypes.c_uint32]
        self._ntt2d = L._Z16ntt_parallel2D_hPjPKjjjjjyij
        self._ntt2d.argtypes = [_u32p, _u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint32]
        self._mpoly = L._Z12mpoly_eval_hPv
        self._montmult = L._Z10montmult_hPjPKjS1_j

    def msm(self, scl, pts_aff, ec2=0, order=6, max_threads=0):
        scl = np.ascontiguousarray(scl, dtype=np.uint32).reshape(-1)
        pts = np.ascontiguousarray(pts_aff, dtype=np.uint32).reshape(-1)
        n = scl.size // 8
        out = np.zeros(32 if ec2 else 16, dtype=np.uint32)
        a = _JacaddReduced(out.ctypes.data, scl.ctypes.data, pts.ctypes.data, n, 1 if ec2 else 0,
                           0, None, 0, max_threads, 0, 0, 0, 0, 0, 0, order, None)
        self._msm(ctypes.byref(a))
        return out

    def ntt(self, A, roots, levels, astride=1, rstride=1, direction=1, pidx=1):
        A = np.array(A, dtype=np.uint32, copy=True).reshape(-1, 8)
        roots = np.ascontiguousarray(roots, dtype=np.uint32)
        self._ntt(_p(A), _p(roots), levels, astride, rstride, direction, pidx)
        return A

    def intt(self, A, roots, levels, rstride=1, fmat=1, pidx=1):
        A = np.array(A, dtype=np.uint32, copy=True).reshape(-1, 8)
        roots = np.ascontiguousarray(roots, dtype=np.uint32)
        self._intt(_p(A), _p(roots), fmat, levels, rstride, pidx)
        return A

    def ntt_parallel(self, A, roots, nrows, ncols, rstride=1, direction=1, fft_mode=0, pidx=1):
        """ntt_parallel_h (src/cuda/ntt.cpp:274): four-step transform of 2^(nrows+ncols)."""
        A = np.array(A, dtype=np.uint32, copy=True).reshape(-1, 8)
        roots = np.ascontiguousarray(roots, dtype=np.uint32)
        self._nttp(_p(A), _p(roots), nrows, ncols, rstride, direction, fft_mode, pidx)
        return A

    def ntt_parallel2D(self, A, roots, nrows, fft_ny, ncols, fft_nx, rstride=1, direction=1, pidx=1):
        """ntt_parallel2D_h (src/cuda/ntt.cpp:199)."""
        A = np.array(A, dtype=np.uint32, copy=True).reshape(-1, 8)
        roots = np.ascontiguousarray(roots, dtype=np.uint32)
        self._ntt2d(_p(A), _p(roots), nrows, fft_ny, ncols, fft_nx, rstride, direction, pidx)
        return A

    def mmul(self, levels):
        """get_Mmul_h (src/cuda/ntt.cpp:650) after an interpolandmul of 2^levels points."""
        ptr = self._mmul()
        return np.ctypeslib.as_array(ptr, shape=((2 << levels) * 8,)).copy().reshape(-1, 8)

    def interpolandmul(self, A, B, roots_full, levels, rstride=2, max_threads=8):
        """roots_full: the caller's concatenated table [2m | 2^(n/2) | 2^(...)] roots."""
        A = np.array(A, dtype=np.uint32, copy=True).reshape(-1)
        B = np.array(B, dtype=np.uint32, copy=True).reshape(-1)
        roots = np.ascontiguousarray(roots_full, dtype=np.uint32).reshape(-1)
        ncols = levels // 2
        nrows = levels - ncols
        a = _InterpolAndMul(A.ctypes.data, B.ctypes.data, roots.ctypes.data, nrows, ncols, 0, 0,
                            levels, rstride, 1, max_threads, 0, 0, 0)
        ptr = self._interp(ctypes.byref(a))
        M = np.ctypeslib.as_array(ptr, shape=((2 << levels) * 8,)).copy()
        return M.reshape(-1, 8)

    def mpoly_eval(self, scalar, pin, ncoeff, start_idx, last_idx, pidx=1):
        scalar = np.ascontiguousarray(scalar, dtype=np.uint32).reshape(-1)
        pin = np.ascontiguousarray(pin, dtype=np.uint32).reshape(-1)
        out = np.zeros(ncoeff * 8, dtype=np.uint32)
        a = _MpolyEval(out.ctypes.data, scalar.ctypes.data, pin.ctypes.data, 0, start_idx,
                       last_idx, 0, 0, pidx)
        self._mpoly(ctypes.byref(a))
        return out.reshape(-1, 8)

    def montmult(self, a, b, pidx):
        a = np.ascontiguousarray(a, dtype=np.uint32).reshape(-1, 8)
        b = np.ascontiguousarray(b, dtype=np.uint32).reshape(-1, 8)
        z = np.zeros_like(a)
        for i in range(a.shape[0]):
            self._montmult(_p(z[i]), _p(a[i]), _p(b[i]), ctypes.c_uint32(pidx))
        return z


def hstep_roots_table(oracle: Oracle, levels: int) -> np.ndarray:
    """The roots table the reference prover hands to ntt_interpolandmul_h for m = 2^levels
    (groth_prover.py:308-334): [2^(L+1) | 2^floor((L+1)/2) | 2^(...)] decimated roots."""
    nroots = levels + 1
    nroots2 = nroots // 2
    nroots3 = nroots2 + 1 if nroots % 2 else nroots2 - 1
    return np.concatenate([oracle.find_roots(nroots), oracle.find_roots(nroots2),
                           oracle.find_roots(nroots3)])
