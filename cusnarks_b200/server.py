"""Served proving: a continuous-batching prove server over resident proving keys
(C ABI cs_server_*; replaces the reference's single-proof TCP loop, groth_prover.py:808-891).

    srv = ProveServer(device=0, slots=3)
    k = srv.add_key(prover)                 # a groth.Prover: key resident in HBM
    t = srv.submit(k, w, r, s)              # returns at once
    proof, info = srv.wait(t)               # 64 words, {"queue_ms", "latency_ms", "device_ms"}
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import lib, ServerResult, ServerStats, CS_OK, CS_ERR_TIMEOUT, CsError


class ProveServer:
    def __init__(self, device: int = 0, slots: int = 3, reserve_bytes: int = 1 << 30, max_batch: int = 16):
        """max_batch: same-key requests of a small key (at most 2^16 constraints) that one slot
        proves in one batched pass (cs_server_set_max_batch; batches of 4, 8 or 16); below 4 proves
        one at a time."""
        h = ctypes.c_void_p()
        st = lib().cs_server_create(device, slots, reserve_bytes, ctypes.byref(h))
        if st != CS_OK:
            raise CsError(st, "cs_server_create failed")
        self.handle = h
        st = lib().cs_server_set_max_batch(h, max_batch)
        if st != CS_OK:
            lib().cs_server_destroy(h)
            self.handle = None
            raise CsError(st, "cs_server_set_max_batch failed")
        self._keys = []
        self._pending = {}

    def add_key(self, prover) -> int:
        kid = ctypes.c_int()
        st = lib().cs_server_add_key(self.handle, prover.handle, ctypes.byref(kid))
        if st != CS_OK:
            raise CsError(st, "cs_server_add_key failed")
        self._keys.append(prover)   # the key must outlive the server
        return kid.value

    def submit(self, key: int, w, r, s) -> int:
        w = np.ascontiguousarray(w, dtype=np.uint32)
        r = np.ascontiguousarray(r, dtype=np.uint32).reshape(8)
        s = np.ascontiguousarray(s, dtype=np.uint32).reshape(8)
        proof = np.zeros(64, dtype=np.uint32)
        t = ctypes.c_uint64()
        st = lib().cs_server_submit(self.handle, key, w.ctypes.data, r.ctypes.data, s.ctypes.data,
                                    proof.ctypes.data, ctypes.byref(t))
        if st != CS_OK:
            raise CsError(st, "cs_server_submit failed")
        self._pending[t.value] = (w, proof)   # buffers stay alive until wait()
        return t.value

    def wait(self, ticket: int, timeout: float = -1.0):
        """Blocks until the proof is done; returns (proof, info).  Raises on failure; on a
        timeout raises TimeoutError and the request stays pending."""
        res = ServerResult()
        st = lib().cs_server_wait(self.handle, ticket, timeout, ctypes.byref(res))
        if st == CS_ERR_TIMEOUT:
            raise TimeoutError(f"proof {ticket} still pending")
        w, proof = self._pending.pop(ticket)
        if st != CS_OK:
            msg = lib().cs_server_error(self.handle)
            raise CsError(st, msg.decode() if msg else "prove failed")
        return proof, {"queue_ms": res.queue_ms, "latency_ms": res.latency_ms, "device_ms": res.device_ms}

    def cancel(self, ticket: int) -> bool:
        """Removes a still-queued request; its wait() then raises CsError(CS_ERR_CANCELLED)."""
        return lib().cs_server_cancel(self.handle, ticket) == CS_OK

    def stats(self) -> dict:
        s = ServerStats()
        lib().cs_server_stats(self.handle, ctypes.byref(s))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def close(self):
        if getattr(self, "handle", None):
            lib().cs_server_destroy(self.handle)
            self.handle = None
            self._pending.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
