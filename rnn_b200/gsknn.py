"""ctypes bindings of libgsknn.so.

Mirrors the reference's Python wrapper (python/gsknn.py:10-183): the four functions
``sgsknn``, ``dgsknn``, ``sgsknn_ref`` and ``dgsknn_ref`` take

    (d, k, Xq, Xq2, q, Xr, Xr2, r, D, I)

with ``Xq``/``Xr`` the query/reference point tables (row-major, N x d), ``Xq2``/``Xr2`` their
squared norms, ``q``/``r`` int32 index arrays of the queries and references, and ``D``/``I`` the
(len(q), k) neighbour heaps, updated in place. They call the same C entry points the reference
wrapper binds (``*_var1`` for the fused path, ``*_ref`` for the reference algorithm).

Differences from the reference wrapper: the library is the in-tree rnn_b200/libgsknn.so (the
reference loads $GSKNN_DIR/lib/libgsknn.so on every call); the size check is
``D.size == n * k`` (the reference asserts ``n * d``, python/gsknn.py:21-22, which only holds
when d == k); a failed call raises ``GsknnError`` with the library's message.

``knn_device`` runs the same pipeline on torch CUDA tensors without host copies.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgsknn.so")

_lib = None
_lock = threading.Lock()

MODE_AUTO, MODE_FP32, MODE_TF32, MODE_BF16 = 0, 1, 2, 3
EARLY_RETURN = 1
KNN_2NORM, KNN_1NORM = 0, 1  # knn_type (include/gsknn.h)


class GsknnError(RuntimeError):
    pass


class HeapT(ctypes.Structure):
    """heap_t (include/gsknn.h)."""
    _fields_ = [("m", ctypes.c_int), ("k", ctypes.c_int), ("ldk", ctypes.c_int),
                ("d", ctypes.c_int), ("ro", ctypes.c_double),
                ("D", ctypes.POINTER(ctypes.c_double)), ("ro_s", ctypes.c_float),
                ("D_s", ctypes.POINTER(ctypes.c_float)), ("I", ctypes.POINTER(ctypes.c_int)),
                ("type", ctypes.c_int), ("prec", ctypes.c_int)]


EXPORTED = [
    "sgsknn", "dgsknn", "sgsknn_var1", "dgsknn_var1", "dgsknn_var3", "dgssq2nrm",
    "gsknn_malloc_aligned", "heapCreate_s", "heapCreate_d", "heapFree_s", "heapFree_d",
    "heapAttach_s", "heapAttach_d", "heapSelect_s", "heapSelect_d", "heapSelect_dheap",
    "swap_float", "swap_double", "swap_int", "bubbleSort_s", "bubbleSort_d", "sgsknn_ref",
    "dgsknn_ref", "gsknn_last_error", "gsknn_last_error_string", "gsknn_set_mode",
    "gsknn_get_mode", "gsknn_s_device", "gsknn_d_device", "gsknn_stream_status",
    "gsknn_release_workspace",
]


def lib():
    """Load (building first if needed and possible) the in-tree libgsknn.so."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                from rnn_b200 import build as _b
                _b.build()
            L = ctypes.CDLL(LIB_PATH)
            L.gsknn_last_error_string.restype = ctypes.c_char_p
            for nm in ("heapCreate_s", "heapCreate_d", "heapAttach_s", "heapAttach_d"):
                getattr(L, nm).restype = ctypes.POINTER(HeapT)
            L.heapCreate_s.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float]
            L.heapCreate_d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
            L.gsknn_malloc_aligned.restype = ctypes.c_void_p
            ll, vp, ci = ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int
            for nm in ("gsknn_s_device", "gsknn_d_device"):
                getattr(L, nm).argtypes = [ci, ci, ci, ci, vp, vp, ll, vp, vp, vp, ll, vp, vp,
                                           vp, ci, vp]
            L.gsknn_stream_status.argtypes = [vp]
            _lib = L
        return _lib


def last_error():
    L = lib()
    return L.gsknn_last_error(), L.gsknn_last_error_string().decode()


def _raise_on_error(allow_early=True):
    code, msg = last_error()
    if code == 0 or (allow_early and code == EARLY_RETURN):
        return
    raise GsknnError(f"gsknn error {code}: {msg}")


def set_mode(mode: int) -> None:
    lib().gsknn_set_mode(ctypes.c_int(mode))
    _raise_on_error()


def get_mode() -> int:
    return lib().gsknn_get_mode()


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _check(d, k, Xq, Xq2, q, Xr, Xr2, r, D, I, dtype):
    M = Xr.shape[0]
    N = Xq.shape[0]
    m = r.size
    n = q.size
    assert Xr.shape[1] == Xq.shape[1] == d
    assert M >= m
    assert N >= n
    assert Xq2.size == N
    assert Xr2.size == M
    assert D.size == n * k
    assert I.size == n * k
    for a in (Xq, Xr, Xq2, Xr2, D):
        assert a.dtype == dtype
    for a in (q, r, I):
        assert a.dtype == numpy.int32
    for a in (Xq, Xr, Xq2, Xr2, q, r, D, I):
        assert a.flags["C_CONTIGUOUS"]
    return m, n


def sgsknn(d, k, Xq, Xq2, q, Xr, Xr2, r, D, I):
    m, n = _check(d, k, Xq, Xq2, q, Xr, Xr2, r, D, I, numpy.float32)
    lib().sgsknn_var1(ctypes.c_int(n), ctypes.c_int(m), ctypes.c_int(d), ctypes.c_int(k),
                      _p(Xq), _p(Xq2), _p(q), _p(Xr), _p(Xr2), _p(r), _p(D), _p(I))
    _raise_on_error()


def dgsknn(d, k, Xq, Xq2, q, Xr, Xr2, r, D, I):
    m, n = _check(d, k, Xq, Xq2, q, Xr, Xr2, r, D, I, numpy.double)
    lib().dgsknn_var1(ctypes.c_int(n), ctypes.c_int(m), ctypes.c_int(d), ctypes.c_int(k),
                      _p(Xq), _p(Xq2), _p(q), _p(Xr), _p(Xr2), _p(r), _p(D), _p(I))
    _raise_on_error()


def sgsknn_ref(d, k, Xq, Xq2, q, Xr, Xr2, r, D, I):
    m, n = _check(d, k, Xq, Xq2, q, Xr, Xr2, r, D, I, numpy.float32)
    lib().sgsknn_ref(ctypes.c_int(m), ctypes.c_int(n), ctypes.c_int(d), ctypes.c_int(k),
                     _p(Xr), _p(Xr2), _p(r), _p(Xq), _p(Xq2), _p(q), _p(D), _p(I))
    _raise_on_error()


def dgsknn_ref(d, k, Xq, Xq2, q, Xr, Xr2, r, D, I):
    m, n = _check(d, k, Xq, Xq2, q, Xr, Xr2, r, D, I, numpy.double)
    lib().dgsknn_ref(ctypes.c_int(m), ctypes.c_int(n), ctypes.c_int(d), ctypes.c_int(k),
                     _p(Xr), _p(Xr2), _p(r), _p(Xq), _p(Xq2), _p(q), _p(D), _p(I))
    _raise_on_error()


# ---- heap_t helpers --------------------------------------------------------------------
class Heap:
    """Owning wrapper of a library heap_t (heapCreate_s/d); numpy views of its storage."""

    def __init__(self, n, k, ro=None, double=True):
        L = lib()
        self.double = double
        if ro is None:
            ro = 1.79e308 if double else 1.79e30
        self.ptr = L.heapCreate_d(n, k, ro) if double else L.heapCreate_s(n, k, ro)
        if not self.ptr:
            raise GsknnError("heapCreate failed")
        h = self.ptr.contents
        self.n, self.k, self.ldk, self.arity = h.m, h.k, h.ldk, h.d
        src = h.D if double else h.D_s
        self.D = numpy.ctypeslib.as_array(src, shape=(self.n, self.ldk))
        self.I = numpy.ctypeslib.as_array(h.I, shape=(self.n, self.ldk))

    @property
    def type(self) -> int:
        """heap_t.type: KNN_2NORM (default) or KNN_1NORM, the distance of calls on this heap."""
        return self.ptr.contents.type

    @type.setter
    def type(self, t: int) -> None:
        self.ptr.contents.type = int(t)

    def free(self):
        if self.ptr:
            (lib().heapFree_d if self.double else lib().heapFree_s)(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def gsknn_heap(k, XA, XA2, alpha, XB, XB2, beta, heap: Heap):
    """dgsknn / sgsknn(m=|alpha|, n=|beta|, d, k, XA, XA2, alpha, XB, XB2, beta, heap)."""
    L = lib()
    f = L.dgsknn if heap.double else L.sgsknn
    f(ctypes.c_int(alpha.size), ctypes.c_int(beta.size), ctypes.c_int(XA.shape[1]),
      ctypes.c_int(k), _p(XA), _p(XA2), _p(alpha), _p(XB), _p(XB2), _p(beta), heap.ptr)
    _raise_on_error()


def dgssq2nrm(XA, XA2, amap, XB, XB2, bmap, ldc=None):
    """C[j, i] = squared distance between XA[amap[i]] and XB[bmap[j]] (n x ldc, float64)."""
    m, n = amap.size, bmap.size
    ldc = m if ldc is None else ldc
    C = numpy.zeros((n, ldc), dtype=numpy.float64)
    lib().dgssq2nrm(ctypes.c_int(m), ctypes.c_int(n), ctypes.c_int(XA.shape[1]), _p(XA),
                    _p(XA2), _p(amap), _p(XB), _p(XB2), _p(bmap), _p(C), ctypes.c_int(ldc))
    _raise_on_error()
    return C


# ---- device tensors (torch) -------------------------------------------------------------
def knn_device(XA, XA2, alpha, XB, XB2, beta, D, I, stream=None, check=True,
               metric=KNN_2NORM):
    """Fused kNN on CUDA tensors: m = len(alpha) candidates of table XA, n = len(beta) queries
    of table XB; D/I (n, k) heaps on the device, updated in place, asynchronously on `stream`
    (default: torch's current stream). With `check`, synchronises and raises on a device-side
    error (an index outside its table). `metric` KNN_1NORM selects the 1-norm
    (gsknn_*_device_metric); its norms XA2 / XB2 are not read and may be None."""
    import torch
    L = lib()
    assert D.dim() == 2 and I.shape == D.shape
    n, k = D.shape
    d = XA.shape[1]
    dt = XA.dtype
    for t in (XA, XA2, XB, XB2, D):
        assert (t is None and metric == KNN_1NORM) or (
            t.dtype == dt and t.is_cuda and t.is_contiguous())
    for t in (alpha, beta, I):
        assert t.dtype == torch.int32 and t.is_cuda and t.is_contiguous()
    assert beta.numel() == n and XB.shape[1] == d
    st = torch.cuda.current_stream(XA.device) if stream is None else stream
    ptr = (lambda t: 0 if t is None else t.data_ptr())
    args = (alpha.numel(), n, d, k, XA.data_ptr(), ptr(XA2), XA.shape[0], alpha.data_ptr(),
            XB.data_ptr(), ptr(XB2), XB.shape[0], beta.data_ptr(), D.data_ptr(), I.data_ptr(),
            D.stride(0), st.cuda_stream)
    if metric == KNN_2NORM:
        f = L.gsknn_s_device if dt == torch.float32 else L.gsknn_d_device
        rc = f(*args)
    else:
        f = L.gsknn_s_device_metric if dt == torch.float32 else L.gsknn_d_device_metric
        ll, vp, ci = ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int
        f.argtypes = [ci, ci, ci, ci, ci, vp, vp, ll, vp, vp, vp, ll, vp, vp, vp, ci, vp]
        rc = f(metric, *args)
    if rc not in (0, EARLY_RETURN):
        _raise_on_error(False)
    if check:
        if L.gsknn_stream_status(ctypes.c_void_p(st.cuda_stream)) != 0:
            _raise_on_error(False)


# ---- sorted-output adapters (frame/old/dgsrnn_directKQuery.cpp) ----------------------------
def direct_kquery(ref, query, k):
    """dgsrnn_directKQuery (frame/old/dgsrnn_directKQuery.cpp:14-135) on numpy tables: the k
    nearest rows of `ref` (n x dim) for every row of `query` (m x dim), as (dist, id) arrays of
    shape (m, k), each row ascending by (distance, id); ids int64, -1 past n. float64 tables run
    the double library path, float32 the single one."""
    L = lib()
    ref = numpy.ascontiguousarray(ref)
    query = numpy.ascontiguousarray(query)
    assert ref.dtype == query.dtype and ref.dtype in (numpy.float32, numpy.float64)
    assert ref.ndim == query.ndim == 2 and ref.shape[1] == query.shape[1]
    n, dim = ref.shape
    m = query.shape[0]
    dist = numpy.empty((m, k), dtype=ref.dtype)
    ids = numpy.empty((m, k), dtype=numpy.int64)
    f = L.gsknn_direct_kquery_d if ref.dtype == numpy.float64 else L.gsknn_direct_kquery_s
    cl = ctypes.c_long
    rc = f(_p(ref), _p(query), cl(n), cl(m), cl(k), cl(dim), _p(dist), _p(ids))
    if rc not in (0, EARLY_RETURN):
        _raise_on_error(False)
    return dist, ids


def direct_kquery_maps(query, XA2, amap, ref, XB2, bmap, k):
    """dgsrnn_directKQuery_var2 (frame/old/dgsrnn_directKQuery.cpp:141-222): queries amap of
    `query` (norms XA2) against references bmap of `ref` (norms XB2); (dist, id) arrays of
    shape (len(amap), k) left in heap order, as the reference copies them out."""
    L = lib()
    dt = query.dtype
    for a in (query, XA2, ref, XB2):
        assert a.dtype == dt and a.flags["C_CONTIGUOUS"]
    for a in (amap, bmap):
        assert a.dtype == numpy.int32 and a.flags["C_CONTIGUOUS"]
    m, n = amap.size, bmap.size
    dist = numpy.empty((m, k), dtype=dt)
    ids = numpy.empty((m, k), dtype=numpy.int64)
    f = L.gsknn_direct_kquery_maps_d if dt == numpy.float64 else L.gsknn_direct_kquery_maps_s
    ci = ctypes.c_int
    rc = f(ci(m), ci(n), ci(query.shape[1]), ci(k), _p(query), _p(XA2), _p(amap), _p(ref),
           _p(XB2), _p(bmap), _p(dist), _p(ids))
    if rc not in (0, EARLY_RETURN):
        _raise_on_error(False)
    return dist, ids


def heap_sort_device(D, I, stream=None):
    """Sort the heap rows of device tensors D / I (n, k) in place into ascending (distance, id)
    lists (gsknn_heap_sort_*_device), asynchronously on `stream` (default: torch's current)."""
    import torch
    L = lib()
    assert D.dim() == 2 and I.shape == D.shape and D.is_cuda and I.dtype == torch.int32
    assert D.stride(1) == 1 and I.stride(1) == 1 and D.stride(0) == I.stride(0)
    st = torch.cuda.current_stream(D.device) if stream is None else stream
    f = L.gsknn_heap_sort_s_device if D.dtype == torch.float32 else L.gsknn_heap_sort_d_device
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p]
    rc = f(D.data_ptr(), I.data_ptr(), D.shape[0], D.shape[1], D.stride(0), st.cuda_stream)
    if rc not in (0, EARLY_RETURN):
        _raise_on_error(False)
