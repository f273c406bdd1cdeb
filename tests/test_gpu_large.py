"""GPU tests of the explicit-distance path: dgsknn with k > KNN_VAR_THRES (4-ary heaps with the
3-slot header, frame/gsknn.c:597-659), dgssq2nrm (frame/gsknn.c:481-594), the reference-algorithm
entry points sgsknn_ref/dgsknn_ref (frame/gsknn_ref.c) and any k beyond the fused kernels."""
import numpy as np
import pytest

from knn_check import compare_sets, exact_dists, is_maxheap, sorted_rows
from rnn_b200 import gsknn as G
from rnn_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _filled_region(D, I, k):
    f = I[:, 1]
    return [(D[j, 3 + k - f[j]:3 + k], I[j, 3 + k - f[j]:3 + k]) for j in range(D.shape[0])]


def test_var3_k600_against_reference(oracle, golden):
    """Three merging calls (300, 500, 1024 candidates) into heapCreate_d(n=32, k=600): partial
    fill, fill completion, replacement -- the reference library's own outputs (golden)."""
    g = golden("var3_k600")
    k, X, X2, beta = int(g["k"]), g["X"], g["X2"], g["beta"]
    h = G.Heap(beta.size, k, 1.79e308, double=True)
    assert h.arity == 4
    Do, Io = g["Din"].copy(), g["Iin"].copy()
    for c, m in enumerate(g["ms"]):
        alpha = np.ascontiguousarray(g["alphas"][c][:m])
        G.gsknn_heap(k, X, X2, alpha, X, X2, beta, h)
        oracle.dgsknn_var3(k, X, X2, alpha, X, X2, beta, Do, Io)
        D, I = np.array(h.D), np.array(h.I)
        # header: k, filled count, ldk
        assert np.array_equal(I[:, :3], g["Iouts"][c][:, :3]), f"call {c}"
        assert oracle.is_maxheap4(np.ascontiguousarray(D), np.ascontiguousarray(I), k)
        got = _filled_region(D, I, k)
        ref = _filled_region(g["Douts"][c], g["Iouts"][c], k)
        for j in range(beta.size):
            gd, gi = got[j]
            rd, ri = ref[j]
            assert np.array_equal(np.sort(gi), np.sort(ri)), f"call {c} row {j}"
            assert np.allclose(np.sort(gd), np.sort(rd), rtol=1e-12, atol=1e-13)
        # unfilled slots keep the creation sentinels
        f = I[:, 1]
        for j in range(beta.size):
            assert np.all(D[j, 3:3 + k - f[j]] == 1.79e308)
    h.free()


def test_dgssq2nrm_against_reference(golden):
    g = golden("dgssq2nrm_d300")
    X, X2, amap, bmap, ldc = g["X"], g["X2"], g["amap"], g["bmap"], int(g["ldc"])
    C = G.dgssq2nrm(X, X2, amap, X, X2, bmap, ldc=ldc)
    ref = g["C"]
    scale = X2[amap][None, :] + X2[bmap][:, None]
    assert np.all(np.abs(C[:, :amap.size] - ref) <= 1e-14 * scale + 1e-15)
    assert np.all(C[:, amap.size:] == 0.0)  # columns beyond m are not written


@pytest.mark.parametrize("case", ["ref_d_basic", "ref_s_basic", "ref_d_prefill", "ref_s_gmm_d64",
                                  "ref_d_few", "ref_d_odd", "ref_s_odd", "ref_d_one"])
def test_ref_entry_points(oracle, golden, case):
    """sgsknn_ref / dgsknn_ref through the python wrapper (python/gsknn.py:10-53, 99-143)."""
    g = golden(case)
    X, X2, alpha, beta, k = g["X"], g["X2"], g["alpha"], g["beta"], int(g["k"])
    D, I = g["Din"].copy(), g["Iin"].copy()
    f = G.dgsknn_ref if X.dtype == np.float64 else G.sgsknn_ref
    f(X.shape[1], k, X, X2, beta, X, X2, alpha, D, I)
    assert is_maxheap(D)
    De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta, g["Din"], g["Iin"])
    eps = 1e-12 if X.dtype == np.float64 else 4e-6
    band = eps * np.maximum(1.0, np.abs(De).max(axis=1)) * 16
    eq, bad = compare_sets(I, Ie, De, band,
                           dist_of=lambda j, ids: exact_dists(X, beta[j], ids, X2))
    assert not bad, bad[:5]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("k", [257, 600, 2000])
def test_large_k_binary(oracle, dtype, k):
    """k beyond the fused kernels' lists, through *_var1 (binary heaps)."""
    N, d = 5000, 24
    X = W.uniform_table(900 + k, N, d, dtype)
    X2 = W.sq_norms(X)
    alpha = W.permutation(901, N)[:3000].astype(np.int32)
    beta = W.permutation(902, N)[:150].astype(np.int32)
    big = 1.79e308 if dtype == np.float64 else 1.79e30
    D = np.full((150, k), big, dtype=dtype)
    I = np.full((150, k), -1, dtype=np.int32)
    prev = G.get_mode()
    G.set_mode(G.MODE_FP32)
    try:
        f = G.dgsknn if dtype == np.float64 else G.sgsknn
        f(d, k, X, X2, beta, X, X2, alpha, D, I)
    finally:
        G.set_mode(prev)
    assert is_maxheap(D)
    De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta, np.full((150, k), big, dtype=dtype),
                              np.full((150, k), -1, dtype=np.int32))
    eps = 1e-12 if dtype == np.float64 else 4e-6
    band = eps * np.maximum(1.0, np.abs(De).max(axis=1)) * 16
    eq, bad = compare_sets(I, Ie, De, band,
                           dist_of=lambda j, ids: exact_dists(X, beta[j], ids, X2))
    assert not bad, bad[:5]


def test_large_k_fewer_candidates_than_k(oracle):
    """k = 700 with 400 candidates: sentinels stay in the binary heap rows."""
    N, d, k = 1000, 10, 700
    X = W.uniform_table(950, N, d)
    X2 = W.sq_norms(X)
    alpha = W.permutation(951, N)[:400].astype(np.int32)
    beta = W.permutation(952, N)[:40].astype(np.int32)
    D = np.full((40, k), 1.79e308)
    I = np.full((40, k), -1, dtype=np.int32)
    G.dgsknn(d, k, X, X2, beta, X, X2, alpha, D, I)
    assert np.all((I >= 0).sum(axis=1) == 400)
    assert is_maxheap(D)
    De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta, np.full((40, k), 1.79e308),
                              np.full((40, k), -1, dtype=np.int32))
    Ds, Is = sorted_rows(D, I)
    assert np.array_equal(Is, Ie)


@pytest.mark.parametrize("case", ["ref_d_stl", "ref_d_basic", "ref_s_basic"])
def test_ref_stl_entry_points(oracle, golden, case):
    """sgsknn_ref_stl / dgsknn_ref_stl through the C ABI (frame/gsknn_ref_stl.cpp): the same sets
    as the exact oracle, and on the STL fixture as the reference's own STL oracle, modulo ties at
    the k-th distance; rows are valid max-heaps."""
    import ctypes
    g = golden(case)
    X, X2, alpha, beta, k = g["X"], g["X2"], g["alpha"], g["beta"], int(g["k"])
    D, I = g["Din"].copy(), g["Iin"].copy()
    L = G.lib()
    f = L.dgsknn_ref_stl if X.dtype == np.float64 else L.sgsknn_ref_stl
    ci = ctypes.c_int
    f(ci(alpha.size), ci(beta.size), ci(X.shape[1]), ci(k), G._p(X), G._p(X2), G._p(alpha),
      G._p(X), G._p(X2), G._p(beta), G._p(D), G._p(I))
    assert G.last_error()[0] == 0
    assert is_maxheap(D)
    De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta, g["Din"], g["Iin"])
    eps = 1e-12 if X.dtype == np.float64 else 4e-6
    band = eps * np.maximum(1.0, np.abs(De).max(axis=1)) * 16
    dist_of = lambda j, ids: exact_dists(X, beta[j], ids, X2)  # noqa: E731
    eq, bad = compare_sets(I, Ie, De, band, dist_of=dist_of)
    assert not bad, bad[:5]
    if case == "ref_d_stl":  # the reference STL oracle's own rows
        Ds, Is = sorted_rows(g["Dout"], g["Iout"])
        eq, bad = compare_sets(I, Is, Ds, band, dist_of=dist_of)
        assert not bad, bad[:5]
