"""ctypes loader for the parity checkers. TEST INFRASTRUCTURE ONLY.

Two libraries are exposed, both built by oracle/Makefile:

* ``liboracle.so``          -- this repository's C restatement of the reference algorithm
                               (oracle/gsknn_oracle.c);
* ``_ref/libgsknn_ref.so``  -- the reference GSKNN library compiled from its own sources; it
                               exists where the reference sources were present at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgsknn_ref.so")

_vp = ctypes.c_void_p
_i = ctypes.c_int


def _p(a):
    return None if a is None else _vp(a.ctypes.data)


def _check(a, dtype, name):
    if a is None:
        return
    if a.dtype != dtype or not a.flags["C_CONTIGUOUS"]:
        raise TypeError(f"{name}: expected contiguous {np.dtype(dtype)}, got {a.dtype}")


def build(ref: bool = False) -> None:
    """Build liboracle.so (and the reference library when `ref` and its sources exist)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


class Oracle:
    """The C restatement (liboracle.so)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)

    def set_threads(self, n: int) -> None:
        self.lib.oracle_set_threads(_i(n))

    # -- reference routines restated ------------------------------------------------------
    def heap_select(self, x, alpha, D, I):
        f = self.lib.oracle_heap_select_d if x.dtype == np.float64 else self.lib.oracle_heap_select_s
        f(_i(x.size), _i(D.size), _p(x), _p(alpha), _p(D), _p(I))

    def gsknn_ref(self, k, XA, XA2, alpha, XB, XB2, beta, D, I):
        """dgsknn_ref / sgsknn_ref semantics: D/I are (n, k), updated in place."""
        dt = XA.dtype
        for a, nm in ((XA, "XA"), (XA2, "XA2"), (XB, "XB"), (XB2, "XB2"), (D, "D")):
            _check(a, dt, nm)
        for a, nm in ((alpha, "alpha"), (beta, "beta"), (I, "I")):
            _check(a, np.int32, nm)
        f = self.lib.oracle_dgsknn_ref if dt == np.float64 else self.lib.oracle_sgsknn_ref
        f(_i(alpha.size), _i(beta.size), _i(XA.shape[1]), _i(k), _p(XA), _p(XA2), _p(alpha),
          _p(XB), _p(XB2), _p(beta), _p(D), _p(I))

    def dgssq2nrm(self, XA, XA2, amap, XB, XB2, bmap, ldc=None):
        m, n, d = amap.size, bmap.size, XA.shape[1]
        ldc = m if ldc is None else ldc
        C = np.zeros((n, ldc), dtype=np.float64)
        self.lib.oracle_dgssq2nrm(_i(m), _i(n), _i(d), _p(XA), _p(XA2), _p(amap), _p(XB),
                                  _p(XB2), _p(bmap), _p(C), _i(ldc))
        return C

    def heapselect_d4(self, key, val, D, I, k):
        self.lib.oracle_heapselect_d4(_i(key.size), _i(k), _p(key), _p(val), _p(D), _p(I))

    def dgsknn_var3(self, k, XA, XA2, alpha, XB, XB2, beta, D, I):
        """D/I are heap_t storage (n, ldk) with the 3-slot header; updated in place."""
        self.lib.oracle_dgsknn_var3(_i(alpha.size), _i(beta.size), _i(XA.shape[1]), _i(k),
                                    _p(XA), _p(XA2), _p(alpha), _p(XB), _p(XB2), _p(beta),
                                    _p(D), _p(I), _i(D.shape[1]))

    # -- tie-resolved exact selection -----------------------------------------------------
    def knn_exact(self, k, XA, XA2, alpha, XB, XB2, beta, Din=None, Iin=None, clamp=True):
        """Sorted k nearest (FP64 distances, lower index wins ties), merged with Din/Iin."""
        n = beta.size
        Dout = np.empty((n, k), dtype=np.float64)
        Iout = np.empty((n, k), dtype=np.int32)
        f = self.lib.oracle_knn_exact_d if XA.dtype == np.float64 else self.lib.oracle_knn_exact_s
        ldin = 0 if Din is None else Din.shape[1]
        f(_i(alpha.size), _i(n), _i(XA.shape[1]), _i(k), _p(XA), _p(XA2), _p(alpha), _p(XB),
          _p(XB2), _p(beta), _p(Din), _p(Iin), _i(ldin), _i(1 if clamp else 0), _p(Dout),
          _p(Iout))
        return Dout, Iout

    def knn_exact_l1(self, k, XA, alpha, XB, beta, Din=None, Iin=None):
        """Sorted k nearest in the 1-norm (in-order sums in the input precision, lower index
        wins ties), merged with Din/Iin."""
        n = beta.size
        Dout = np.empty((n, k), dtype=np.float64)
        Iout = np.empty((n, k), dtype=np.int32)
        f = (self.lib.oracle_knn_exact_l1_d if XA.dtype == np.float64
             else self.lib.oracle_knn_exact_l1_s)
        ldin = 0 if Din is None else Din.shape[1]
        f(_i(alpha.size), _i(n), _i(XA.shape[1]), _i(k), _p(XA), _p(alpha), _p(XB), _p(beta),
          _p(Din), _p(Iin), _i(ldin), _p(Dout), _p(Iout))
        return Dout, Iout

    def select_rows(self, C, alpha, k, Din=None, Iin=None):
        n, ldc = C.shape
        Dout = np.empty((n, k), dtype=np.float64)
        Iout = np.empty((n, k), dtype=np.int32)
        ldin = 0 if Din is None else Din.shape[1]
        self.lib.oracle_select_rows_d(_i(alpha.size), _i(n), _i(k), _p(C), _i(ldc), _p(alpha),
                                      _p(Din), _p(Iin), _i(ldin), _p(Dout), _p(Iout))
        return Dout, Iout

    def allnn_leaves(self, k, X, X2, ptr, pts, Din=None, Iin=None):
        """Batching form: per point, the k nearest among its leaf-mates (all leaves given)
        and its incoming heap row; FP64, sorted ascending, lower id first on ties."""
        N, d = X.shape
        Dout = np.empty((N, k), dtype=np.float64)
        Iout = np.empty((N, k), dtype=np.int32)
        ptr = np.ascontiguousarray(ptr, dtype=np.int32)
        pts = np.ascontiguousarray(pts, dtype=np.int32)
        ldin = 0 if Din is None else Din.shape[1]
        self.lib.oracle_allnn_leaves_s(_i(N), _i(d), _i(k), _p(X), _p(X2), _i(ptr.size - 1),
                                       _p(ptr), _p(pts), _p(Din), _p(Iin), _i(ldin), _p(Dout),
                                       _p(Iout))
        return Dout, Iout

    def heap_pop_rows(self, D, I, k=None):
        """Ascending (dist, id int64) lists popped from max-heap rows D / I (copies consumed),
        as dgsrnn_directKQuery does (frame/old/dgsrnn_directKQuery.cpp:112-124)."""
        n, ld = D.shape
        k = ld if k is None else k
        D = np.ascontiguousarray(D).copy()
        I = np.ascontiguousarray(I, dtype=np.int32).copy()
        Dout = np.empty((n, k), dtype=D.dtype)
        Iout = np.empty((n, k), dtype=np.int64)
        f = (self.lib.oracle_heap_pop_rows_d if D.dtype == np.float64
             else self.lib.oracle_heap_pop_rows_s)
        f(_i(n), _i(k), _i(ld), _p(D), _p(I), _p(Dout), _p(Iout))
        return Dout, Iout

    def is_maxheap(self, D, k=None):
        n, ld = D.shape
        k = ld if k is None else k
        f = self.lib.oracle_is_maxheap_d if D.dtype == np.float64 else self.lib.oracle_is_maxheap_s
        return bool(f(_i(n), _i(k), _i(ld), _p(D)))

    def is_maxheap4(self, D, I, k):
        n, ld = D.shape
        return bool(self.lib.oracle_is_maxheap4_d(_i(n), _i(k), _i(ld), _p(D), _p(I)))


class HeapT(ctypes.Structure):
    """heap_t (include/gsknn.h:75-88 of the reference)."""
    _fields_ = [("m", ctypes.c_int), ("k", ctypes.c_int), ("ldk", ctypes.c_int),
                ("d", ctypes.c_int), ("ro", ctypes.c_double),
                ("D", ctypes.POINTER(ctypes.c_double)), ("ro_s", ctypes.c_float),
                ("D_s", ctypes.POINTER(ctypes.c_float)), ("I", ctypes.POINTER(ctypes.c_int)),
                ("type", ctypes.c_int), ("prec", ctypes.c_int)]


class ReferenceLib:
    """The reference GSKNN library compiled from its sources (oracle/_ref/libgsknn_ref.so)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.lib.heapCreate_d.restype = ctypes.POINTER(HeapT)
        self.lib.heapCreate_s.restype = ctypes.POINTER(HeapT)
        self.lib.heapCreate_d.argtypes = [_i, _i, ctypes.c_double]
        self.lib.heapCreate_s.argtypes = [_i, _i, ctypes.c_float]

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def gsknn_ref(self, k, XA, XA2, alpha, XB, XB2, beta, D, I, stl=False):
        dt = XA.dtype
        name = ("dgsknn_ref" if dt == np.float64 else "sgsknn_ref") + ("_stl" if stl else "")
        getattr(self.lib, name)(_i(alpha.size), _i(beta.size), _i(XA.shape[1]), _i(k), _p(XA),
                                _p(XA2), _p(alpha), _p(XB), _p(XB2), _p(beta), _p(D), _p(I))

    def var1(self, k, Xq, Xq2, q, Xr, Xr2, r, D, I):
        """{d,s}gsknn_var1(n=|q|, m=|r|, ...) exactly as python/gsknn.py:79-92 calls it."""
        f = self.lib.dgsknn_var1 if Xq.dtype == np.float64 else self.lib.sgsknn_var1
        f(_i(q.size), _i(r.size), _i(Xq.shape[1]), _i(k), _p(Xq), _p(Xq2), _p(q), _p(Xr),
          _p(Xr2), _p(r), _p(D), _p(I))

    def heap_create(self, n, k, ro, double=True):
        if double:
            return self.lib.heapCreate_d(n, k, ro)
        return self.lib.heapCreate_s(n, k, ro)

    def heap_arrays(self, h, double=True):
        hh = h.contents
        rows, ld = hh.m, hh.ldk
        if double:
            D = np.ctypeslib.as_array(hh.D, shape=(rows, ld))
        else:
            D = np.ctypeslib.as_array(hh.D_s, shape=(rows, ld))
        I = np.ctypeslib.as_array(hh.I, shape=(rows, ld))
        return D, I

    def heap_free(self, h, double=True):
        (self.lib.heapFree_d if double else self.lib.heapFree_s)(h)

    def gsknn(self, k, XA, XA2, alpha, XB, XB2, beta, h):
        """dgsknn / sgsknn(m=|alpha|, n=|beta|, d, k, ..., heap)."""
        f = self.lib.dgsknn if XA.dtype == np.float64 else self.lib.sgsknn
        f(_i(alpha.size), _i(beta.size), _i(XA.shape[1]), _i(k), _p(XA), _p(XA2), _p(alpha),
          _p(XB), _p(XB2), _p(beta), h)

    def dgssq2nrm(self, XA, XA2, amap, XB, XB2, bmap, ldc=None):
        m, n, d = amap.size, bmap.size, XA.shape[1]
        ldc = ((m + 7) // 8) * 8 if ldc is None else ldc
        # The reference kernel stores 8x4 tiles with aligned vector stores (sq2nrm_asm_d8x4.c);
        # allocate padded, 32-byte aligned storage the way gsknn_malloc_aligned does.
        ncols = ((n + 3) // 4) * 4 + 4
        raw = np.zeros(ldc * ncols + 8, dtype=np.float64)
        off = (-raw.ctypes.data % 32) // 8
        C = raw[off:off + ldc * ncols].reshape(ncols, ldc)
        self.lib.dgssq2nrm(_i(m), _i(n), _i(d), _p(XA), _p(XA2), _p(amap), _p(XB), _p(XB2),
                           _p(bmap), _p(C), _i(ldc))
        return np.array(C[:n])

    def heap_select(self, x, alpha, D, I):
        f = self.lib.heapSelect_d if x.dtype == np.float64 else self.lib.heapSelect_s
        f(_i(x.size), _i(D.size), _p(x), _p(alpha), _p(D), _p(I))
