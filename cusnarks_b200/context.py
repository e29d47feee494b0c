"""Python face of the context API (cs_* in include/cusnarks_b200.h).

``Context`` owns a cs_ctx (one CUDA stream, scratch arena, timing events).  Host-array
methods take numpy uint32 arrays in the reference layout (8 limbs per field element) and
return numpy arrays; ``*_device`` methods take raw device pointers (for example
``torch.Tensor.data_ptr()``) and run asynchronously on the context stream.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import lib, check


def _as_u32(a, cols=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    if cols is not None:
        a = a.reshape(-1, cols)
    return a


class Context:
    def __init__(self, device: int = 0):
        self._lib = lib()
        h = ctypes.c_void_p()
        check(self._lib.cs_ctx_create(device, ctypes.byref(h)))
        self.handle = h
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            self._lib.cs_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ plumbing ----
    def set_stream(self, stream_handle: int):
        """Run device-pointer calls on an existing cudaStream_t (e.g. torch's)."""
        check(self._lib.cs_ctx_set_stream(self.handle, ctypes.c_void_p(stream_handle)), self.handle)

    def sync(self):
        check(self._lib.cs_ctx_sync(self.handle), self.handle)

    def set_prove_graphs(self, enable: bool):
        """Capture and replay each key's proof launch sequence as a CUDA graph (default on)."""
        check(self._lib.cs_ctx_set_prove_graphs(self.handle, int(bool(enable))), self.handle)

    def set_msm_affine_rounds(self, rounds: int):
        """Batch-affine halving rounds before the XYZZ bucket accumulation (-1 auto, 0 off)."""
        check(self._lib.cs_ctx_set_msm_affine_rounds(self.handle, rounds), self.handle)

    @property
    def last_ms(self) -> float:
        return float(self._lib.cs_ctx_last_ms(self.handle))

    @property
    def last_phase_ms(self) -> float:
        """Device ms of the bucket-accumulation kernels of the last MSM."""
        return float(self._lib.cs_ctx_last_phase_ms(self.handle))

    # ------------------------------------------------------------------------ MSM ----
    def msm(self, scalars, points, ec2: bool = False, window: int = 0) -> np.ndarray:
        """sum_i scalars[i] * points[i]; affine Montgomery result (16 or 32 words)."""
        pw = 32 if ec2 else 16
        s = _as_u32(scalars, 8)
        p = _as_u32(points, pw)
        if s.shape[0] != p.shape[0]:
            raise ValueError("scalars and points differ in length")
        out = np.zeros(pw, dtype=np.uint32)
        check(self._lib.cs_msm(self.handle, int(bool(ec2)), s.ctypes.data, p.ctypes.data,
                               s.shape[0], out.ctypes.data, window), self.handle)
        return out

    def msm_device(self, d_scalars: int, d_points: int, n: int, d_out: int, ec2: bool = False,
                   window: int = 0):
        check(self._lib.cs_msm_device(self.handle, int(bool(ec2)), ctypes.c_void_p(d_scalars),
                                      ctypes.c_void_p(d_points), n, ctypes.c_void_p(d_out), window),
              self.handle)

    @staticmethod
    def msm_workspace_bytes(n: int, ec2: bool = False, window: int = 0) -> int:
        return int(lib().cs_msm_workspace_bytes(n, int(bool(ec2)), window))

    # ---------------------------------------------------- fixed-base (resident) MSM ----
    @staticmethod
    def msm_fixed_window(n: int, ec2: bool = False) -> int:
        return int(lib().cs_msm_fixed_window(n, int(bool(ec2))))

    @staticmethod
    def msm_fixed_table_points(n: int, window: int) -> int:
        return int(lib().cs_msm_fixed_table_points(n, window))

    def msm_fixed_table_device(self, d_points: int, n: int, window: int, d_table: int, ec2: bool = False):
        """d_table (msm_fixed_table_points(n, window) affine points) <- 2^(window j) P_i."""
        check(self._lib.cs_msm_fixed_table_device(self.handle, int(bool(ec2)), ctypes.c_void_p(d_points), n,
                                                  window, ctypes.c_void_p(d_table)), self.handle)

    def msm_fixed_device(self, d_scalars: int, d_table: int, n: int, window: int, d_out: int,
                         ec2: bool = False):
        check(self._lib.cs_msm_fixed_device(self.handle, int(bool(ec2)), ctypes.c_void_p(d_scalars),
                                            ctypes.c_void_p(d_table), n, window, ctypes.c_void_p(d_out)),
              self.handle)

    # ----------------------------------------------------------------- batched MSM ----
    def msm_batch(self, jobs, ec2: bool = False, task: int = 0) -> "MsmBatch":
        """jobs: [(d_scalars, d_points, n, d_out[, window])] device pointers -> a batch plan."""
        return MsmBatch(self, jobs, ec2, task)

    def msm_autotune(self, log_min: int, log_max: int, ec2: bool = False) -> list:
        out = (ctypes.c_int * (log_max - log_min + 1))()
        check(self._lib.cs_msm_autotune(self.handle, int(bool(ec2)), log_min, log_max, out), self.handle)
        return list(out)

    def msm_tuned_window(self, n: int, ec2: bool = False) -> int:
        return int(self._lib.cs_msm_tuned_window(self.handle, int(bool(ec2)), n))

    # -------------------------------------------------------------- field ops -----
    FOP = {"mul": 0, "add": 1, "sub": 2, "sqr": 3, "inv": 4, "to_mont": 5, "from_mont": 6,
           "fq2_mul": 8, "mul_dp52": 9}

    def field_op_device(self, op: str, pidx: int, d_a: int, d_b: int, d_out: int, n: int):
        check(self._lib.cs_field_op_device(self.handle, self.FOP[op], pidx, ctypes.c_void_p(d_a),
                                           ctypes.c_void_p(d_b or 0), ctypes.c_void_p(d_out), n),
              self.handle)

    # ------------------------------------------------------------ transforms ------
    def ntt_device(self, d_in: int, d_out: int, log_n: int, direction: int = 1, fmat: int = 1):
        check(self._lib.cs_ntt_device(self.handle, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out),
                                      log_n, direction, fmat), self.handle)

    def hstep_device(self, variant: int, d_a: int, d_b: int, d_c: int, log_m: int, d_out: int):
        """variant 0: reference (2m coefficients of A*B); 1: coset quotient (m coefficients)."""
        check(self._lib.cs_hstep_device(self.handle, variant, ctypes.c_void_p(d_a), ctypes.c_void_p(d_b),
                                        ctypes.c_void_p(d_c or 0), log_m, ctypes.c_void_p(d_out)),
              self.handle)

    # ------------------------------------------------------------- scalar mult ----
    def scmul_device(self, d_scalars: int, d_points: int, n: int, d_out: int, ec2: bool = False,
                     point_stride_words: int | None = None):
        """out[i] = scalars[i] * points[i]; point_stride_words=0 for one shared base."""
        if point_stride_words is None:
            point_stride_words = 32 if ec2 else 16
        check(self._lib.cs_scmul_device(self.handle, int(bool(ec2)), ctypes.c_void_p(d_scalars),
                                        ctypes.c_void_p(d_points), point_stride_words, n,
                                        ctypes.c_void_p(d_out)), self.handle)

    def point_sum_device(self, d_points: int, n: int, d_out: int, ec2: bool = False, dims: int = 2):
        """d_out = the affine sum of n points (rows of dims = 2 affine / 3 Jacobian coordinates)."""
        check(self._lib.cs_point_sum_device(self.handle, int(bool(ec2)), ctypes.c_void_p(d_points), n, dims,
                                            ctypes.c_void_p(d_out)), self.handle)

    def pipe_rate(self, mode: int) -> float:
        """Measured instruction rate per second of one pipe probe (cs_bench_pipe): 1 mad.lo,
        2 mad.hi, 3 mad.wide.u32 (one 32x32->64 product each), 5 carry-chain mad.cc."""
        v = ctypes.c_double()
        check(self._lib.cs_bench_pipe(self.handle, mode, ctypes.byref(v)), self.handle)
        return float(v.value)


class MsmBatch:
    """A batch of MSM instances summed in one pass (cs_msm_batch_*)."""

    def __init__(self, ctx: Context, jobs, ec2: bool = False, task: int = 0):
        from ._lib import MsmJob
        arr = (MsmJob * max(1, len(jobs)))()
        for k, j in enumerate(jobs):
            w = j[4] if len(j) > 4 else 0
            arr[k] = MsmJob(ctypes.c_void_p(j[0]), ctypes.c_void_p(j[1]), ctypes.c_void_p(j[3]), j[2], w)
        h = ctypes.c_void_p()
        check(lib().cs_msm_batch_create(ctx.handle, int(bool(ec2)), ctypes.cast(arr, ctypes.c_void_p), len(jobs),
                                        task, ctypes.byref(h)), ctx.handle)
        self.ctx, self.handle, self.njobs = ctx, h, len(jobs)

    def run(self, graph: bool = True):
        check(lib().cs_msm_batch_run(self.ctx.handle, self.handle, int(bool(graph))), self.ctx.handle)

    def windows(self) -> list:
        return [int(lib().cs_msm_batch_window(self.handle, k)) for k in range(self.njobs)]

    def workspace_bytes(self) -> int:
        return int(lib().cs_msm_batch_workspace_bytes(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            lib().cs_msm_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kernel_launches() -> int:
    return int(lib().cs_kernel_launches())
