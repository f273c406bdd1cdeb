"""GPU parity of the 1-norm variant (kernels/x86_64/sandybridge/rnn_r_1norm_int_d8x4_row.c):
heap_t.type = KNN_1NORM through sgsknn / dgsknn / dgsknn_var3, and gsknn_*_device_metric.

Bars:
  * against the reference kernel's own heaps (tests/golden/l1_*.npz): distances bit for bit,
    index sets equal except at exact ties on the k-th distance (the reference keeps the later
    candidate, this library the lower id);
  * against the oracle's restatement (in-order sums in the input precision, ties to the lower
    id): identical sorted rows, in double and in float, for the fused lists (k <= 256) and the
    explicit-distance path beyond;
  * heaps merge across calls; rows are valid max-heaps (4-ary with header for dgsknn_var3).
"""
import numpy as np
import pytest

from knn_check import is_maxheap, sorted_rows
from rnn_b200 import gsknn as G
from rnn_b200 import workloads as W

pytestmark = pytest.mark.gpu

DMAX = np.finfo(np.float64).max


@pytest.mark.parametrize("case", ["l1_d_basic", "l1_d_ties", "l1_d_odd", "l1_d_few",
                                  "l1_d_dim1"])
def test_dgsknn_l1_heap_matches_reference_kernel(oracle, golden, case):
    g = golden(case)
    k, XQ, XC = int(g["k"]), g["XQ"], g["XC"]
    m, n = XQ.shape[0], XC.shape[0]
    h = G.Heap(m, k, ro=DMAX, double=True)
    h.type = G.KNN_1NORM
    alpha = np.arange(n, dtype=np.int32)
    beta = np.arange(m, dtype=np.int32)
    G.gsknn_heap(k, XC, W.sq_norms(XC), alpha, XQ, W.sq_norms(XQ), beta, h)
    D, I = h.D[:, :k].copy(), h.I[:, :k].copy()
    h.free()
    assert is_maxheap(D)
    Ds, Is = sorted_rows(D, I)
    Rs, Ri = sorted_rows(g["Dout"], g["Iout"])
    assert np.array_equal(Ds, Rs)  # bit for bit
    De, Ie = oracle.knn_exact_l1(k, XC, alpha, XQ, beta, g["Din"], g["Iin"])
    assert np.array_equal(Ds, De) and np.array_equal(Is, Ie)
    if case != "l1_d_ties":
        assert np.array_equal(Is, Ri)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("k", [1, 8, 32, 100, 256, 300, 700])
def test_device_metric_l1_against_oracle(oracle, dtype, k):
    torch = pytest.importorskip("torch")
    N, d = 6000, 19
    X = W.uniform_table(400 + k, N, d).astype(dtype)
    alpha = W.permutation(401 + k, N)[:3000].astype(np.int32)
    beta = W.permutation(402 + k, N)[:777].astype(np.int32)
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    Xt = torch.from_numpy(X).cuda()
    at = torch.from_numpy(alpha).cuda()
    bt = torch.from_numpy(beta).cuda()
    D = torch.full((beta.size, k), float("inf"), dtype=tdt, device="cuda")
    I = torch.full((beta.size, k), -1, dtype=torch.int32, device="cuda")
    G.knn_device(Xt, None, at, Xt, None, bt, D, I, metric=G.KNN_1NORM)  # norms not needed
    Dh, Ih = D.cpu().numpy(), I.cpu().numpy()
    assert is_maxheap(Dh)
    De, Ie = oracle.knn_exact_l1(k, X, alpha, X, beta)
    Ds, Is = sorted_rows(Dh, Ih)
    assert np.array_equal(Ds.astype(np.float64), De)
    assert np.array_equal(Is, Ie)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_l1_heap_merges_across_calls(oracle, dtype):
    """Two calls over disjoint candidate halves into one heap equal one call over all."""
    N, d, k = 4000, 12, 24
    X = W.uniform_table(410, N, d).astype(dtype)
    X2 = W.sq_norms(X)
    alpha = W.permutation(411, N)[:2400].astype(np.int32)
    beta = W.permutation(412, N)[:300].astype(np.int32)
    h = G.Heap(beta.size, k, double=dtype == np.float64)
    h.type = G.KNN_1NORM
    for part in (alpha[:1200], alpha[1200:]):
        G.gsknn_heap(k, X, X2, np.ascontiguousarray(part), X, X2, beta, h)
    Ds, Is = sorted_rows(h.D[:, :k].copy(), h.I[:, :k].copy())
    h.free()
    De, Ie = oracle.knn_exact_l1(k, X, alpha, X, beta)
    assert np.array_equal(Ds.astype(np.float64), De) and np.array_equal(Is, Ie)


def test_dgsknn_var3_l1_four_ary(oracle):
    """k > 512 in double: dgsknn goes to dgsknn_var3 over the 4-ary heap with its header."""
    N, d, k = 3000, 9, 600
    X = W.uniform_table(420, N, d)
    X2 = W.sq_norms(X)
    alpha = W.permutation(421, N)[:2000].astype(np.int32)
    beta = W.permutation(422, N)[:64].astype(np.int32)
    h = G.Heap(beta.size, k, double=True)
    assert h.arity == 4
    h.type = G.KNN_1NORM
    G.gsknn_heap(k, X, X2, alpha, X, X2, beta, h)
    off = 3  # KNN_HEAP_OFFSET: D = [ro, 0, 0 | heap], I = [k, filled, ldk | heap]
    assert np.all(h.I[:, 0] == k) and np.all(h.I[:, 1] == k)
    Ds, Is = sorted_rows(h.D[:, off:off + k].copy(), h.I[:, off:off + k].copy())
    assert oracle.is_maxheap4(h.D.copy(), h.I.copy(), k)
    h.free()
    De, Ie = oracle.knn_exact_l1(k, X, alpha, X, beta)
    assert np.array_equal(Ds, De) and np.array_equal(Is, Ie)


def test_l1_type_leaves_l2_untouched(oracle):
    """A heap of the default type still gets squared 2-norm distances."""
    N, d, k = 2000, 8, 10
    X = W.uniform_table(430, N, d)
    X2 = W.sq_norms(X)
    alpha = np.arange(N, dtype=np.int32)
    beta = np.arange(50, dtype=np.int32)
    h = G.Heap(beta.size, k, double=True)
    assert h.type == G.KNN_2NORM
    G.gsknn_heap(k, X, X2, alpha, X, X2, beta, h)
    Ds, Is = sorted_rows(h.D[:, :k].copy(), h.I[:, :k].copy())
    h.free()
    De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta)
    assert np.array_equal(Is, Ie)
