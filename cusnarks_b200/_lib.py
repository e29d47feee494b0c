"""ctypes binding of libcusnarks_b200.so (declarations: include/cusnarks_b200.h).

The library is the product: every call here runs CUDA kernels.  There is no CPU
fallback -- if the shared library is missing or cannot be loaded, ``lib()`` raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libcusnarks_b200.so")

CS_OK = 0
CS_ERR_CUDA = 1
CS_ERR_ARG = 2
CS_ERR_NOMEM = 3
CS_ERR_UNSUPPORTED = 4
CS_ERR_NODEVICE = 5
CS_ERR_TIMEOUT = 6
CS_ERR_CANCELLED = 7

_u32p = ctypes.POINTER(ctypes.c_uint32)
_vp = ctypes.c_void_p


class CsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cusnarks_b200 error {code}: {msg}")
        self.code = code


class MsmJob(ctypes.Structure):
    _fields_ = [("scalars", _vp), ("points", _vp), ("out", _vp), ("n", ctypes.c_uint32), ("window", ctypes.c_int)]


class ServerResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("queue_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("device_ms", ctypes.c_float)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64), ("rejected", ctypes.c_uint64),
                ("cancelled", ctypes.c_uint64), ("queued", ctypes.c_uint64), ("running", ctypes.c_uint32),
                ("max_concurrent", ctypes.c_uint32), ("promised_bytes", ctypes.c_size_t),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("hbm_free_bytes", ctypes.c_size_t), ("hbm_total_bytes", ctypes.c_size_t),
                ("batched", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("max_batch_seen", ctypes.c_uint32)]


class MpolyEval(ctypes.Structure):
    """mpoly_eval_t (reference src/cuda/types.h:516-528)."""
    _fields_ = [("pout", _vp), ("scalar", _vp), ("pin", _vp), ("reduce_coeff", ctypes.c_uint32),
                ("start_idx", ctypes.c_uint32), ("last_idx", ctypes.c_uint32),
                ("max_threads", ctypes.c_uint32), ("thread_id", ctypes.c_uint32), ("pidx", ctypes.c_uint32)]


class PkDesc(ctypes.Structure):
    """cs_pk_desc (include/cusnarks_b200.h)."""
    _fields_ = [("n_vars", ctypes.c_uint32), ("n_public", ctypes.c_uint32), ("domain_size", ctypes.c_uint32),
                ("polsA", _vp), ("polsA_words", ctypes.c_size_t), ("polsA_entries", ctypes.c_uint32),
                ("polsB", _vp), ("polsB_words", ctypes.c_size_t), ("polsB_entries", ctypes.c_uint32),
                ("A", _vp), ("B1", _vp), ("B2", _vp), ("C", _vp), ("hExps", _vp), ("delta_1", _vp)]


class InterpolAndMul(ctypes.Structure):
    """ntt_interpolandmul_t (reference src/cuda/types.h:530-546)."""
    _fields_ = [("A", _vp), ("B", _vp), ("roots", _vp), ("Nrows", ctypes.c_uint32),
                ("Ncols", ctypes.c_uint32), ("mNrows", ctypes.c_uint32), ("mNcols", ctypes.c_uint32),
                ("nroots", ctypes.c_uint32), ("rstride", ctypes.c_uint32), ("pidx", ctypes.c_uint32),
                ("max_threads", ctypes.c_uint32), ("start_idx", ctypes.c_uint32),
                ("last_idx", ctypes.c_uint32), ("thread_id", ctypes.c_uint32)]


class JacaddReduced(ctypes.Structure):
    """jacadd_reduced_t (reference src/cuda/types.h:548-567)."""
    _fields_ = [("out_ep", _vp), ("scl", _vp), ("x", _vp), ("n", ctypes.c_uint32),
                ("ec2", ctypes.c_uint32), ("compute_table", ctypes.c_uint32), ("ec_table", _vp),
                ("pidx", ctypes.c_uint32), ("max_threads", ctypes.c_uint32),
                ("start_idx", ctypes.c_uint32), ("last_idx", ctypes.c_uint32),
                ("thread_id", ctypes.c_uint32), ("pippen", ctypes.c_uint32),
                ("offset", ctypes.c_uint64), ("total_words", ctypes.c_uint64),
                ("order", ctypes.c_uint32), ("filename", ctypes.c_char_p)]


# (name, restype, argtypes)
_SIGNATURES = [
    ("cs_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    ("cs_ctx_destroy", None, [_vp]),
    ("cs_ctx_set_stream", ctypes.c_int, [_vp, _vp]),
    ("cs_ctx_stream", _vp, [_vp]),
    ("cs_ctx_sync", ctypes.c_int, [_vp]),
    ("cs_ctx_error", ctypes.c_char_p, [_vp]),
    ("cs_ctx_last_ms", ctypes.c_float, [_vp]),
    ("cs_ctx_last_phase_ms", ctypes.c_float, [_vp]),
    ("cs_last_status", ctypes.c_int, []),
    ("cs_last_error", ctypes.c_char_p, []),
    ("cs_msm", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_uint32, _vp, ctypes.c_int]),
    ("cs_msm_device", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_uint32, _vp, ctypes.c_int]),
    ("cs_msm_workspace_bytes", ctypes.c_size_t, [ctypes.c_uint32, ctypes.c_int, ctypes.c_int]),
    ("cs_msm_default_window", ctypes.c_int, [ctypes.c_uint32, ctypes.c_int]),
    ("cs_msm_num_windows", ctypes.c_int, [ctypes.c_int]),
    ("cs_ctx_set_msm_affine_rounds", ctypes.c_int, [_vp, ctypes.c_int]),
    ("cs_ctx_prove_stages", ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    ("cs_ctx_set_prove_graphs", ctypes.c_int, [_vp, ctypes.c_int]),
    ("cs_msm_fixed_window", ctypes.c_int, [ctypes.c_uint32, ctypes.c_int]),
    ("cs_msm_fixed_table_points", ctypes.c_size_t, [ctypes.c_uint32, ctypes.c_int]),
    ("cs_msm_fixed_workspace_bytes", ctypes.c_size_t, [ctypes.c_uint32, ctypes.c_int, ctypes.c_int]),
    ("cs_msm_fixed_table_device", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_uint32, ctypes.c_int, _vp]),
    ("cs_msm_fixed_device", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_uint32, ctypes.c_int, _vp]),
    ("cs_msm_batch_create", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(_vp)]),
    ("cs_msm_batch_run", ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    ("cs_msm_batch_destroy", None, [_vp]),
    ("cs_msm_batch_workspace_bytes", ctypes.c_size_t, [_vp]),
    ("cs_msm_batch_window", ctypes.c_int, [_vp, ctypes.c_uint32]),
    ("cs_msm_autotune", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, _vp]),
    ("cs_msm_tuned_window", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_uint32]),
    ("cs_scmul_device", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_uint32, ctypes.c_uint32, _vp]),
    ("cs_point_sum_device", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_uint32, ctypes.c_int, _vp]),
    ("cs_bench_pipe", ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    ("cs_kernel_launches", ctypes.c_ulonglong, []),
    ("cs_field_op_device", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, ctypes.c_uint32]),
    ("cs_field_last_status", ctypes.c_int, []),
    ("montmult_h", None, [_vp, _vp, _vp, ctypes.c_uint32]),
    ("montsquare_h", None, [_vp, _vp, ctypes.c_uint32]),
    ("addm_h", None, [_vp, _vp, _vp, ctypes.c_uint32]),
    ("subm_h", None, [_vp, _vp, _vp, ctypes.c_uint32]),
    ("montinv_h", None, [_vp, _vp, ctypes.c_uint32]),
    ("to_montgomeryN_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32]),
    ("from_montgomeryN_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("ntt_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_int32, ctypes.c_uint32]),
    ("intt_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_ulonglong, ctypes.c_uint32]),
    ("find_roots_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32]),
    ("ntt_interpolandmul_server_h", ctypes.POINTER(ctypes.c_uint32), [_vp]),
    ("get_Mtranspose_h", ctypes.POINTER(ctypes.c_uint32), []),
    ("get_Mmul_h", ctypes.POINTER(ctypes.c_uint32), []),
    ("ntt_parallel_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_ulonglong, ctypes.c_int32,
                              ctypes.c_int, ctypes.c_uint32]),
    ("ntt_parallel2D_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                ctypes.c_ulonglong, ctypes.c_int32, ctypes.c_uint32]),
    ("cs_ntt_last_status", ctypes.c_int, []),
    ("cs_ntt_device", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_uint32, ctypes.c_int, ctypes.c_int]),
    ("cs_hstep_device", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, ctypes.c_uint32, _vp]),
    ("cs_msm_g1_noalloc", ctypes.c_int, [_vp, _vp, ctypes.c_uint32, _vp, _vp]),
    ("cs_msm_noalloc_scratch_bytes", ctypes.c_size_t, []),
    ("cs_msm_g1_noalloc_max_terms", ctypes.c_uint32, []),
    ("cs_msm_g1_noalloc_error", ctypes.c_char_p, []),
    ("mpoly_eval_server_h", None, [_vp]),
    ("mpoly_eval_h", _vp, [_vp]),
    ("cs_qap_last_status", ctypes.c_int, []),
    ("cs_pk_create", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    ("cs_pk_destroy", None, [_vp]),
    ("cs_prove_workspace_bytes", ctypes.c_size_t, [_vp]),
    ("cs_pk_fixed_base", ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    ("cs_pk_device_bytes", ctypes.c_size_t, [_vp]),
    ("cs_pk_fixed_window", ctypes.c_int, [_vp, ctypes.c_int]),
    ("cs_prove", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    ("cs_prove_device", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    ("cs_prove_batch_device", ctypes.c_int, [_vp, _vp, ctypes.c_uint32, _vp, _vp, _vp, _vp]),
    ("cs_server_create", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(_vp)]),
    ("cs_server_destroy", None, [_vp]),
    ("cs_server_add_key", ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_int)]),
    ("cs_server_submit", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_uint64)]),
    ("cs_server_wait", ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(ServerResult)]),
    ("cs_server_stats", ctypes.c_int, [_vp, ctypes.POINTER(ServerStats)]),
    ("cs_server_error", ctypes.c_char_p, [_vp]),
    ("cs_server_cancel", ctypes.c_int, [_vp, ctypes.c_uint64]),
    ("cs_server_set_max_batch", ctypes.c_int, [_vp, ctypes.c_int]),
    ("cs_debug_fail_allocs", None, [ctypes.c_int]),
    ("cs_setup_lagrange", ctypes.c_int, [_vp, ctypes.c_uint32, _vp, _vp]),
    ("cs_setup_wire_eval", ctypes.c_int, [_vp, _vp, ctypes.c_uint32, _vp, ctypes.c_uint32, _vp]),
    ("cs_setup_c_scalars", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_uint32, _vp]),
    ("cs_setup_pow_scalars", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_uint32, _vp]),
    ("cs_r1cs_layer_eval", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_uint32, _vp, _vp]),
    ("ec_jacreduce_server_h", None, [ctypes.POINTER(JacaddReduced)]),
    ("ec_jac2aff_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec2_jac2aff_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec_jacaddreduce_h", None, [_vp, _vp] + [ctypes.c_uint32] * 5),
    ("ec2_jacaddreduce_h", None, [_vp, _vp] + [ctypes.c_uint32] * 5),
    ("ec_jacscmul_h", None, [_vp, _vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec2_jacscmul_h", None, [_vp, _vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec_jacsc1mul_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec2_jacsc1mul_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec_isoncurve_h", ctypes.c_uint32, [_vp, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec2_isoncurve_h", ctypes.c_uint32, [_vp, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec_inittable_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec2_inittable_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec_isinf", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec2_isinf", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32]),
    ("ec_jacadd_h", None, [_vp, _vp, _vp, ctypes.c_uint32]),
    ("ec2_jacadd_h", None, [_vp, _vp, _vp, ctypes.c_uint32]),
    ("ec_jacdouble_h", None, [_vp, _vp, ctypes.c_uint32]),
    ("ec2_jacdouble_h", None, [_vp, _vp, ctypes.c_uint32]),
    ("mpoly_from_montgomery_h", None, [_vp, ctypes.c_uint32]),
    ("mpoly_to_montgomery_h", None, [_vp, ctypes.c_uint32]),
    ("addu256_h", None, [_vp, _vp, _vp]),
    ("rangeu256_h", None, [_vp, ctypes.c_uint32, _vp, ctypes.c_uint32, _vp]),
    ("readU256CircuitFileHeader_h", None, [_vp, ctypes.c_char_p]),
    ("readU256PKFileHeader_h", None, [_vp, ctypes.c_char_p]),
    ("sortu256_idx_h", None, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32]),
    ("ntt_build_h", None, [_vp, ctypes.c_uint32]),
    ("init_h", None, []),
    ("release_h", None, []),
    ("get_nprocs_h", ctypes.c_uint32, []),
    ("readU256CircuitFile_h", None, [_vp, ctypes.c_char_p, ctypes.c_ulonglong]),
    ("readU256PKFile_h", None, [_vp, ctypes.c_char_p, ctypes.c_ulonglong]),
    ("readU256DataFile_h", None, [_vp, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32]),
    ("readU256DataFileFromOffset_h", None, [_vp, ctypes.c_char_p, ctypes.c_ulonglong, ctypes.c_ulonglong]),
    ("writeU256DataFile_h", None, [_vp, ctypes.c_char_p, ctypes.c_ulonglong]),
    ("appendU256DataFile_h", None, [_vp, ctypes.c_char_p, ctypes.c_ulonglong]),
    ("readWitnessFile_h", None, [_vp, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_ulonglong]),
    ("writeWitnessFile_h", None, [_vp, ctypes.c_char_p, ctypes.c_ulonglong]),
    ("ec2_jacreduce_server_h", None, [ctypes.POINTER(JacaddReduced)]),
    ("shared_new_h", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_ulonglong]),
    ("shared_free_h", None, [_vp, ctypes.c_int]),
    ("readR1CSFileHeader_h", None, [_vp, ctypes.c_char_p]),
    ("readR1CSFile_h", None, [_vp, ctypes.c_char_p, _vp, ctypes.c_int]),
    ("r1cs_to_mpoly_len_h", None, [_vp, _vp, _vp, ctypes.c_uint32]),
    ("r1cs_to_mpoly_h", None, [_vp, _vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("readECTablesNElementsFile_h", None, [_vp, ctypes.c_char_p]),
]

_lock = threading.Lock()
_lib = None


def exported_symbols():
    return [name for name, _, _ in _SIGNATURES]


def lib() -> ctypes.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m cusnarks_b200.build` "
                    "(nvcc, sm_100a).  There is no CPU fallback.")
            L = ctypes.CDLL(LIB_PATH)
            for name, res, args in _SIGNATURES:
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def check(code: int, ctx=None):
    if code != CS_OK:
        L = lib()
        msg = (L.cs_ctx_error(ctx) if ctx else L.cs_last_error()) or b""
        raise CsError(code, msg.decode(errors="replace"))
