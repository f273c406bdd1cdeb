"""Serving form: kNN requests against a device-resident reference set (C ABI `gsknn_serve_*`).

The reference set is prepared once on the device; requests (m query rows, a k) are queued,
admitted while their result heaps fit the heap budget, packed into batches by a dispatcher
thread inside the library and run on several streams, so requests that arrive while others are
on the GPU start as soon as a stream slot frees (continuous batching). Each request's result is
the exact FP64 top-k of its queries, kept on the device until released.
"""
from __future__ import annotations

import ctypes

import numpy as np

from rnn_b200 import gsknn as G


class Server:
    def __init__(self, R, R2, mode: int = 0, max_batch_queries: int = 8192, max_k: int = 64,
                 heap_budget: int = 1 << 30, slots: int = 3, slice_rows: int = 0):
        """R, R2: CUDA tensors (float32 nref x d, float32 nref), kept alive by the server.
        `slice_rows`: rows per batch (0: sized to a few milliseconds of work)."""
        self._keep = (R, R2)
        self.nref, self.d = R.shape
        L = G.lib()
        vp, ci, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
        L.gsknn_serve_create.restype = vp
        L.gsknn_serve_create.argtypes = [vp, vp, ci, ci, ci, ci, ci, ctypes.c_size_t, ci]
        L.gsknn_serve_submit.restype = ll
        L.gsknn_serve_submit.argtypes = [vp, vp, ci, ci]
        L.gsknn_serve_test.argtypes = [vp, ll]
        L.gsknn_serve_wait.argtypes = [vp, ll, ctypes.c_double]
        L.gsknn_serve_fetch.argtypes = [vp, ll, vp, vp]
        L.gsknn_serve_heap.argtypes = [vp, ll, vp, vp]
        L.gsknn_serve_stats.argtypes = [vp, ll, vp, vp, vp, vp]
        L.gsknn_serve_release.argtypes = [vp, ll]
        L.gsknn_serve_destroy.argtypes = [vp]
        L.gsknn_serve_pause.argtypes = [vp, ci]
        L.gsknn_serve_set_slice.argtypes = [vp, ci]
        self._L = L
        h = L.gsknn_serve_create(R.data_ptr(), R2.data_ptr(), self.nref, self.d, mode,
                                 max_batch_queries, max_k, heap_budget, slots)
        if not h:
            raise G.GsknnError(L.gsknn_last_error(), G.last_error())
        self._h = h
        self._shape = {}
        L.gsknn_serve_mode.argtypes = [vp, vp, vp]
        a, b = ctypes.c_double(0.0), ctypes.c_double(0.0)
        self.mode = L.gsknn_serve_mode(h, ctypes.byref(a), ctypes.byref(b))
        self.probe_ms = {"bf16": a.value, "bf16x3": b.value}
        self.slice_rows = self.set_slice(slice_rows)

    def submit(self, Q: np.ndarray, k: int) -> int:
        Q = np.ascontiguousarray(Q, dtype=np.float32)
        assert Q.ndim == 2 and Q.shape[1] == self.d
        rid = self._L.gsknn_serve_submit(self._h, Q.ctypes.data, Q.shape[0], k)
        if rid < 0:
            raise G.GsknnError(int(-rid), G.last_error())
        self._shape[rid] = (Q.shape[0], k)
        return rid

    def test(self, rid: int) -> int:
        return self._L.gsknn_serve_test(self._h, rid)

    def wait(self, rid: int, timeout: float = 60.0) -> None:
        rc = self._L.gsknn_serve_wait(self._h, rid, timeout)
        if rc != 0:
            raise G.GsknnError(rc, G.last_error())

    def fetch(self, rid: int):
        m, k = self._shape[rid]
        D = np.empty((m, k), dtype=np.float32)
        I = np.empty((m, k), dtype=np.int32)
        rc = self._L.gsknn_serve_fetch(self._h, rid, D.ctypes.data, I.ctypes.data)
        if rc != 0:
            raise G.GsknnError(rc, G.last_error())
        return D, I

    def device_heap(self, rid: int):
        """(D, I) device pointers of a finished request's heap (m x k)."""
        pd, pi = ctypes.c_void_p(), ctypes.c_void_p()
        rc = self._L.gsknn_serve_heap(self._h, rid, ctypes.byref(pd), ctypes.byref(pi))
        if rc != 0:
            raise G.GsknnError(rc, G.last_error())
        return pd.value, pi.value

    def stats(self, rid: int) -> dict:
        q, t = ctypes.c_double(), ctypes.c_double()
        b, r = ctypes.c_int(), ctypes.c_int()
        rc = self._L.gsknn_serve_stats(self._h, rid, ctypes.byref(q), ctypes.byref(t),
                                       ctypes.byref(b), ctypes.byref(r))
        if rc != 0:
            raise G.GsknnError(rc, G.last_error())
        return {"queue_ms": q.value, "total_ms": t.value, "batch": b.value,
                "batch_rows": r.value}

    def release(self, rid: int) -> None:
        rc = self._L.gsknn_serve_release(self._h, rid)
        if rc != 0:
            raise G.GsknnError(rc, G.last_error())
        self._shape.pop(rid, None)

    def set_slice(self, rows: int) -> int:
        """Rows per batch for batches formed from now on (0: the default); returns the value in
        effect."""
        s = self._L.gsknn_serve_set_slice(self._h, int(rows))
        if s <= 0:
            raise G.GsknnError(-s, G.last_error())
        self.slice_rows = s
        return s

    def pause(self, paused: bool = True) -> None:
        """Hold (or resume) the start of new batches; requests keep queueing."""
        self._L.gsknn_serve_pause(self._h, 1 if paused else 0)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.gsknn_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
