"""C-ABI checks that need no GPU: the library loads, exports every function include/gsknn.h
declares, and its host-side utilities (heap_t construction, heapSelect, sorting) behave like
the reference's (fixtures from the reference library in tests/golden/)."""
import ctypes
import os
import re

import numpy as np
import pytest

from rnn_b200 import gsknn as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        txt = re.sub(r"//[^\n]*", "", txt)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(",
                             txt, flags=re.M):
            nm = m.group(1)
            if nm not in ("if", "while", "for", "return", "sizeof"):
                names.append(nm)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = G.lib()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(G.EXPORTED) <= set(names)


def test_early_return_status_without_gpu():
    """m == 0: early return with status 1, D/I untouched (frame/gsknn.c:910-913)."""
    L = G.lib()
    D = np.full(4, 7.0)
    I = np.full(4, -1, dtype=np.int32)
    X = np.zeros((2, 3))
    idx = np.zeros(1, dtype=np.int32)
    L.dgsknn_var1(1, 0, 3, 4, G._p(X), G._p(X[0]), G._p(idx), G._p(X), G._p(X[0]), G._p(idx),
                  G._p(D), G._p(I))
    assert G.last_error()[0] == G.EARLY_RETURN
    assert np.all(D == 7.0) and np.all(I == -1)


def test_heap_create_layouts():
    h = G.Heap(5, 16, 1.79e308, double=True)
    assert (h.ldk, h.arity) == (16, 2)
    assert np.all(h.D == 1.79e308) and np.all(h.I == -1)
    h.free()
    # double heaps with k > KNN_VAR_THRES: 4-ary with a 3-slot header (frame/gsknn_heap.c:257-307)
    h = G.Heap(3, 600, 2.5, double=True)
    assert (h.ldk, h.arity) == (((600 + 2) // 4 + 1) * 4, 4)
    assert np.all(h.D[:, 0] == 2.5) and np.all(h.D[:, 1:3] == 0.0)
    assert np.all(h.I[:, 0] == 600) and np.all(h.I[:, 1] == 0) and np.all(h.I[:, 2] == h.ldk)
    assert np.all(h.D[:, 3:603] == 2.5) and np.all(h.I[:, 3:603] == -1)
    h.free()
    hs = G.Heap(4, 700, 1.0, double=False)  # float heaps are always binary
    assert (hs.ldk, hs.arity) == (700, 2)
    hs.free()


def test_heap_attach():
    L = G.lib()
    D = np.zeros((3, 8))
    I = np.zeros((3, 8), dtype=np.int32)
    p = L.heapAttach_d(3, 8, G._p(D), G._p(I))
    h = p.contents
    assert (h.m, h.k, h.ldk, h.d) == (3, 8, 8, 2)
    assert ctypes.addressof(h.D.contents) == D.ctypes.data


def test_heap_select_matches_reference(golden):
    g = golden("heapselect")
    L = G.lib()
    for tag, f in (("d", L.heapSelect_d), ("s", L.heapSelect_s)):
        D, I = g[f"Din_{tag}"].copy(), g[f"Iin_{tag}"].copy()
        keys, alpha = g[f"keys_{tag}"], g[f"alpha_{tag}"]
        f(keys.size, D.size, G._p(keys), G._p(alpha), G._p(D), G._p(I))
        assert np.array_equal(D, g[f"Dout_{tag}"]) and np.array_equal(I, g[f"Iout_{tag}"])


def test_heap_select_dheap_matches_4ary_reference(oracle):
    rng = np.random.default_rng(5)
    k = 37
    ldk = ((k + 2) // 4 + 1) * 4
    for m in (10, 37, 200):
        D = np.zeros(ldk)
        I = np.zeros(ldk, dtype=np.int32)
        D[0], I[0], I[2] = 9.0, k, ldk
        D[3:3 + k], I[3:3 + k] = 9.0, -1
        D2, I2 = D.copy(), I.copy()
        keys = rng.random(m)
        vals = np.arange(m, dtype=np.int32)
        G.lib().heapSelect_dheap(m, k, G._p(keys), G._p(vals), G._p(D), G._p(I))
        oracle.heapselect_d4(keys, vals, D2, I2, k)
        assert np.array_equal(D, D2) and np.array_equal(I, I2)


def test_bubble_sort():
    L = G.lib()
    D = np.array([3.0, 1.0, 2.0, 1.0])
    I = np.array([0, 1, 2, 3], dtype=np.int32)
    L.bubbleSort_d(4, G._p(D), G._p(I))
    assert list(D) == [1.0, 1.0, 2.0, 3.0] and list(I) == [1, 3, 2, 0]


def test_python_wrapper_checks_shapes():
    X = np.zeros((4, 3), dtype=np.float32)
    X2 = np.zeros(4, dtype=np.float32)
    q = np.arange(2, dtype=np.int32)
    D = np.zeros((2, 5), dtype=np.float32)
    I = np.zeros((2, 5), dtype=np.int32)
    with pytest.raises(AssertionError):
        G.sgsknn(3, 4, X, X2, q, X, X2, q, D, I)  # D is 2 x 5, k = 4
    with pytest.raises(AssertionError):
        G.dgsknn(3, 5, X, X2, q, X, X2, q, D, I)  # float tables to the double entry


def test_sorted_adapters_argument_checks_without_gpu():
    """Early returns and argument errors of the sorted-output adapters are decided on the host
    before any device work."""
    L = G.lib()
    X = np.zeros((2, 3))
    dist = np.zeros(4)
    ids = np.zeros(4, dtype=np.int64)
    cl = ctypes.c_long
    rc = L.gsknn_direct_kquery_d(G._p(X), G._p(X), cl(2), cl(0), cl(2), cl(3), G._p(dist),
                                 G._p(ids))
    assert rc == G.EARLY_RETURN == G.last_error()[0]
    rc = L.gsknn_direct_kquery_d(G._p(X), G._p(X), cl(2), cl(-1), cl(2), cl(3), G._p(dist),
                                 G._p(ids))
    assert rc == 2
    vp, ci = ctypes.c_void_p, ctypes.c_int
    L.gsknn_heap_sort_d_device.argtypes = [vp, vp, ci, ci, ci, vp]
    assert L.gsknn_heap_sort_d_device(None, None, 0, 4, 4, None) == G.EARLY_RETURN
    assert L.gsknn_heap_sort_d_device(None, None, 3, 4, 4, None) == 2
    d = np.zeros(8)
    i = np.zeros(8, dtype=np.int32)
    assert L.gsknn_heap_sort_d_device(G._p(d), G._p(i), 1, 8, 4, None) == 2  # ldk < k
    assert L.gsknn_heap_sort_d_device(G._p(d), G._p(i), 1, 600, 600, None) == 5
    assert "k <= 512" in G.last_error()[1]
