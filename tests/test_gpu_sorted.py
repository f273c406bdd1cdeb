"""GPU parity of the sorted-output adapters (frame/old/dgsrnn_directKQuery.cpp) against the
oracle.

Bars:
  * gsknn_direct_kquery_*: every row ascending; index sets equal the FP64 oracle's modulo ties
    at the k-th distance; double distances within 1e-12 relative of the oracle's; bit-identical
    to the oracle's pops (dgsrnn_directKQuery.cpp:112-124) of the library's own heap rows
    wherever a row has no equal distances; with n < k the tail is (largest finite value, -1);
  * gsknn_direct_kquery_maps_*: the library's heap rows, ids widened to 64 bits;
  * gsknn_heap_sort_*_device: each row equals the host (distance, unsigned id) sort of the same
    heap row, including the order of exact ties, and the oracle's pops where distances differ;
    columns past k of a strided row are untouched.
"""
import numpy as np
import pytest

from knn_check import compare_sets, exact_dists, is_maxheap, sorted_rows
from rnn_b200 import gsknn as G
from rnn_b200 import workloads as W

pytestmark = pytest.mark.gpu


def seq_norms(X):
    """Squared norms summed in order in double, as the adapter computes them."""
    s = np.zeros(X.shape[0])
    for p in range(X.shape[1]):
        c = X[:, p].astype(np.float64)
        s = s + c * c
    return s.astype(X.dtype)


def distinct_rows(D):
    return np.array([np.unique(r).size == r.size for r in D])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("m,n,dim,k", [(300, 5000, 17, 16), (129, 2048, 64, 1),
                                       (64, 3000, 5, 100), (40, 1500, 33, 512)])
def test_direct_kquery_against_oracle(oracle, dtype, m, n, dim, k):
    ref = W.uniform(11, (n, dim)).astype(dtype)
    query = W.uniform(12, (m, dim)).astype(dtype)
    dist, ids = G.direct_kquery(ref, query, k)
    assert dist.shape == (m, k) and ids.dtype == np.int64
    assert np.all(np.diff(dist, axis=1) >= 0)
    r2, q2 = seq_norms(ref), seq_norms(query)
    alpha = np.arange(n, dtype=np.int32)
    beta = np.arange(m, dtype=np.int32)
    De, Ie = oracle.knn_exact(k, ref, r2, alpha, query, q2, beta, clamp=True)
    if dtype == np.float64:
        band = 1e-12 * np.maximum(1.0, De.max(axis=1)) * 8
    else:
        band = 64 * (dim + 4) * 2.0 ** -24 * (q2.astype(np.float64) + r2.max())
    eq, bad = compare_sets(ids.astype(np.int32), Ie, De, band,
                           dist_of=lambda j, c: exact_dists(np.vstack([ref, query]), n + j, c))
    assert not bad, f"{len(bad)} rows differ beyond ties"
    if dtype == np.float64:
        rel = np.abs(dist - De) / np.maximum(np.abs(De), 1.0)
        assert rel.max() <= 1e-12
    # the adapter's own pipeline: the library's heap rows popped as the reference pops them
    Dh, Ih = G.direct_kquery_maps(query, q2, beta, ref, r2, alpha, k)
    assert is_maxheap(Dh)
    Dp, Ip = oracle.heap_pop_rows(Dh, Ih.astype(np.int32))
    keep = distinct_rows(Dh)
    assert keep.mean() > 0.5
    assert np.array_equal(dist[keep], Dp[keep])
    assert np.array_equal(ids[keep], Ip[keep])
    # all rows: the same pairs, ordered by (distance, id)
    Ds, Is = sorted_rows(Dh, Ih.astype(np.int32))
    assert np.array_equal(dist, Ds) and np.array_equal(ids, Is.astype(np.int64))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_direct_kquery_fewer_references_than_k(oracle, dtype):
    """n < k: the rows end with the reference's initial heap entries (largest finite, -1)."""
    m, n, dim, k = 7, 5, 9, 8
    ref = W.uniform(21, (n, dim)).astype(dtype)
    query = W.uniform(22, (m, dim)).astype(dtype)
    dist, ids = G.direct_kquery(ref, query, k)
    big = np.finfo(dtype).max
    assert np.all(ids[:, n:] == -1) and np.all(dist[:, n:] == big)
    De, Ie = oracle.knn_exact(n, ref, seq_norms(ref), np.arange(n, dtype=np.int32), query,
                              seq_norms(query), np.arange(m, dtype=np.int32), clamp=True)
    assert np.array_equal(ids[:, :n], Ie.astype(np.int64))


def test_direct_kquery_reference_test_data(oracle):
    """The reference test's data (test/old/test_dgsrnn_directKQuery.cpp:24-36): coordinates
    (integer in [0, 100)) / 1000, query and reference sets drawn independently; many near
    ties, so index sets are compared modulo ties at the k-th distance."""
    m, n, dim, k = 256, 4096, 8, 32
    query = W.randint(31, m * dim, 100).reshape(m, dim) / 1000.0
    ref = W.randint(32, n * dim, 100).reshape(n, dim) / 1000.0
    dist, ids = G.direct_kquery(ref, query, k)
    assert np.all(np.diff(dist, axis=1) >= 0)
    r2, q2 = seq_norms(ref), seq_norms(query)
    De, Ie = oracle.knn_exact(k, ref, r2, np.arange(n, dtype=np.int32), query, q2,
                              np.arange(m, dtype=np.int32), clamp=True)
    band = 1e-12 * np.maximum(1.0, De.max(axis=1)) * 8
    eq, bad = compare_sets(ids.astype(np.int32), Ie, De, band,
                           dist_of=lambda j, c: exact_dists(np.vstack([ref, query]), n + j, c))
    assert not bad
    rel = np.abs(dist - De) / np.maximum(np.abs(De), 1.0)
    assert rel.max() <= 1e-12


def _device_heaps(torch, dtype, n_q, n_c, dim, k, seed, integer=False):
    if integer:
        X = (W.randint(seed, (n_q + n_c) * dim, 4).reshape(n_q + n_c, dim)).astype(dtype)
    else:
        X = W.uniform(seed, (n_q + n_c, dim)).astype(dtype)
    X2 = seq_norms(X)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    Xt = torch.from_numpy(X).cuda()
    X2t = torch.from_numpy(X2).cuda()
    alpha = torch.arange(n_q, n_q + n_c, dtype=torch.int32, device="cuda")
    beta = torch.arange(n_q, dtype=torch.int32, device="cuda")
    D = torch.full((n_q, k), float("inf"), dtype=tdt, device="cuda")
    I = torch.full((n_q, k), -1, dtype=torch.int32, device="cuda")
    G.knn_device(Xt, X2t, alpha, Xt, X2t, beta, D, I)
    return D, I


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("k", [1, 7, 32, 33, 100, 256, 512])
def test_heap_sort_device(oracle, dtype, k):
    torch = pytest.importorskip("torch")
    D, I = _device_heaps(torch, dtype, 1000, 4000, 24, k, 41 + k)
    Dh, Ih = D.cpu().numpy(), I.cpu().numpy()
    assert is_maxheap(Dh)
    G.heap_sort_device(D, I)
    torch.cuda.synchronize()
    Ds, Is = D.cpu().numpy(), I.cpu().numpy()
    De, Ie = sorted_rows(Dh, Ih)
    assert np.array_equal(Ds, De) and np.array_equal(Is, Ie)
    Dp, Ip = oracle.heap_pop_rows(Dh, Ih)
    keep = distinct_rows(Dh)
    assert np.array_equal(Ds[keep], Dp[keep]) and np.array_equal(Is[keep], Ip[keep])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_heap_sort_device_ties_and_stride(dtype):
    """Small integer coordinates: many exact ties, ordered by id on the device as on the host;
    rows of stride ldk > k keep their columns past k."""
    torch = pytest.importorskip("torch")
    k, ldk = 48, 61
    D, I = _device_heaps(torch, dtype, 517, 3000, 6, k, 51, integer=True)
    Dh, Ih = D.cpu().numpy(), I.cpu().numpy()
    assert not distinct_rows(Dh).all()
    tdt = D.dtype
    Dw = torch.full((517, ldk), -5.0, dtype=tdt, device="cuda")
    Iw = torch.full((517, ldk), -7, dtype=torch.int32, device="cuda")
    Dw[:, :k] = D
    Iw[:, :k] = I
    G.heap_sort_device(Dw[:, :k], Iw[:, :k])
    torch.cuda.synchronize()
    Dw, Iw = Dw.cpu().numpy(), Iw.cpu().numpy()
    De, Ie = sorted_rows(Dh, Ih)
    assert np.array_equal(Dw[:, :k], De) and np.array_equal(Iw[:, :k], Ie)
    assert np.all(Dw[:, k:] == -5.0) and np.all(Iw[:, k:] == -7)


def test_heap_sort_device_padding_rows():
    """Rows with fewer real entries than k (-1 ids at +inf) keep the padding last."""
    torch = pytest.importorskip("torch")
    k = 40
    D, I = _device_heaps(torch, np.float32, 64, 25, 8, k, 61)
    Dh, Ih = D.cpu().numpy(), I.cpu().numpy()
    G.heap_sort_device(D, I)
    torch.cuda.synchronize()
    Ds, Is = D.cpu().numpy(), I.cpu().numpy()
    assert np.all(Is[:, 25:] == -1) and np.all(np.isinf(Ds[:, 25:]))
    De, Ie = sorted_rows(Dh, Ih)
    assert np.array_equal(Ds, De) and np.array_equal(Is, Ie)
