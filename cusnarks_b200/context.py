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

    @property
    def last_ms(self) -> float:
        return float(self._lib.cs_ctx_last_ms(self.handle))

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
