"""GPU parity of the fused kNN path through the C ABI against the oracle.

Bars:
  * double: identical index sets to the FP64 oracle (ties to the lower index), distances within
    1e-12 relative;
  * float: on data whose float arithmetic is exact (small integer coordinates) identical
    (distance, index) rows including the tie rule; on general data every returned distance
    lies within the FP32 rounding bound of the FP64 distance of its id, and index sets equal the
    FP64 oracle's except for ids within that bound of the k-th distance;
  * every output row is a valid binary max-heap (descending order);
  * repeated calls merge with the incoming heap (the reference's in-place contract).
"""
import numpy as np
import pytest

from knn_check import compare_sets, exact_dists, is_maxheap, sorted_rows
from rnn_b200 import gsknn as G
from rnn_b200 import workloads as W

pytestmark = pytest.mark.gpu

EPS32 = 2.0 ** -24


def fp32_bound(X, X2, beta, alpha, d):
    """Per-row absolute error bound of an FP32 squared distance (generous model):
    the dot product, the two norm additions and the -2 scaling, in units of |q|^2 + max|c|^2."""
    qn = X2[beta].astype(np.float64)
    cmax = float(X2[alpha].max()) if alpha.size else 0.0
    return 8.0 * (d + 4) * EPS32 * (qn + cmax + 2.0 * np.sqrt(qn * cmax))


def run_var1(X, X2, alpha, beta, k, Din=None, Iin=None):
    """The python wrapper (python/gsknn.py contract): queries beta, references alpha."""
    n = beta.size
    dt = X.dtype
    if Din is None:
        big = 1.79e308 if dt == np.float64 else 1.79e30
        D = np.full((n, k), big, dtype=dt)
        I = np.full((n, k), -1, dtype=np.int32)
    else:
        D, I = Din.copy(), Iin.copy()
    f = G.dgsknn if dt == np.float64 else G.sgsknn
    f(X.shape[1], k, X, X2, beta, X, X2, alpha, D, I)
    return D, I


def check_against_oracle(oracle, X, X2, alpha, beta, k, D, I, Din, Iin, exact_float=False):
    assert is_maxheap(D), "rows are not max-heaps"
    De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta, Din, Iin, clamp=True)
    Ds, Is = sorted_rows(D.astype(np.float64), I)
    if X.dtype == np.float64 or exact_float:
        eq, bad = compare_sets(I, Ie, De, np.zeros(beta.size))
        assert not bad, f"rows differ: {bad[:8]}"
        if exact_float:
            assert np.array_equal(Is, Ie) and np.array_equal(Ds, De)
        else:
            fin = De < 1e300
            rel = np.abs(Ds[fin] - De[fin]) / np.maximum(np.abs(De[fin]), 1e-300)
            small = De[fin] < 1e-200
            assert np.all((rel <= 1e-12) | (np.abs(Ds[fin] - De[fin]) <= 1e-13 * (1 + De[fin])) | small)
        return
    d = X.shape[1]
    band = fp32_bound(X, X2, beta, alpha, d)
    eq, bad = compare_sets(I, Ie, De, 2 * band,
                           dist_of=lambda j, ids: exact_dists(X, beta[j], ids, X2))
    assert not bad, f"rows differ beyond FP32 rounding: {bad[:8]}"
    # each returned distance matches its id's FP64 distance within the bound
    real = (I >= 0) & (D < 1e29)
    for j in np.nonzero(real.any(axis=1))[0][:512]:
        ids = I[j][real[j]]
        ex = exact_dists(X, beta[j], ids, X2)
        assert np.all(np.abs(D[j][real[j]] - ex) <= band[j] + 1e-30), f"row {j}"


GOLDEN_CASES = ["ref_d_basic", "ref_s_basic", "ref_d_prefill", "ref_s_gmm_d64", "ref_d_ties",
                "ref_s_ties", "ref_d_few", "ref_d_odd", "ref_s_odd", "ref_d_one"]


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_golden_cases(oracle, golden, case):
    g = golden(case)
    X, X2, alpha, beta, k = g["X"], g["X2"], g["alpha"], g["beta"], int(g["k"])
    D, I = run_var1(X, X2, alpha, beta, k, g["Din"], g["Iin"])
    exact_float = "ties" in case
    check_against_oracle(oracle, X, X2, alpha, beta, k, D, I, g["Din"], g["Iin"], exact_float)
    # agreement with the reference's own output, modulo ties (reference keeps later ties)
    if X.dtype == np.float64 and "ties" not in case:
        De, _ = oracle.knn_exact(k, X, X2, alpha, X, X2, beta, g["Din"], g["Iin"])
        eq, bad = compare_sets(I, g["Iout"], De, np.full(beta.size, 1e-12))
        assert not bad


def test_config1_two_calls_heap_api(oracle, golden):
    """Config 1 through dgsknn(heap_t): N=8192, d=32, m=n=4096, k=16, second call merges a
    fresh candidate set into the same heap."""
    g = golden("config1_dgsknn")
    p, alpha2 = W.config1(int(g["seed"]))
    h = G.Heap(p.n, p.k, 1.79e308, double=True)
    G.gsknn_heap(p.k, p.X, p.X2, p.alpha, p.X, p.X2, p.beta, h)
    D1, I1 = h.D.copy(), h.I.copy()
    G.gsknn_heap(p.k, p.X, p.X2, alpha2, p.X, p.X2, p.beta, h)
    D2, I2 = h.D.copy(), h.I.copy()
    h.free()
    D0, I0 = p.empty_heap(1.79e308)
    check_against_oracle(oracle, p.X, p.X2, p.alpha, p.beta, p.k, D1, I1, D0, I0)
    check_against_oracle(oracle, p.X, p.X2, alpha2, p.beta, p.k, D2, I2, D1, I1)
    # the reference library's own results (golden), modulo exact ties
    for (Ig, Ir, Dr) in ((I1, g["I1"], g["D1"]), (I2, g["I2"], g["D2"])):
        eq, bad = compare_sets(Ig, Ir, Dr, np.zeros(p.n))
        assert not bad


SHAPES = [  # (m candidates, n queries, d, k)
    (1, 1, 1, 1), (7, 9, 33, 3), (9, 7, 1, 2), (33, 31, 9, 16), (255, 257, 8, 64),
    (300, 5, 3, 33), (1000, 130, 31, 100), (2000, 70, 64, 128), (3000, 40, 100, 200),
    (4000, 33, 300, 256), (129, 129, 129, 32), (5000, 300, 7, 1),
]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("shape", SHAPES)
def test_shapes(oracle, dtype, shape):
    m, n, d, k = shape
    N = m + n + 17
    X = W.uniform_table(1000 + m + d, N, d, dtype)
    X2 = W.sq_norms(X)
    alpha = W.permutation(7 + m, N)[:m].astype(np.int32)
    beta = W.permutation(9 + n, N)[:n].astype(np.int32)
    D, I = run_var1(X, X2, alpha, beta, k)
    big = 1.79e308 if dtype == np.float64 else 1.79e30
    Din = np.full((n, k), big, dtype=dtype)
    Iin = np.full((n, k), -1, dtype=np.int32)
    check_against_oracle(oracle, X, X2, alpha, beta, k, D, I, Din, Iin)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_integer_grid_ties_exact(oracle, dtype):
    """Small-integer coordinates: float arithmetic is exact, so (distance, index) rows must
    equal the oracle's exactly, including the lower-index tie rule and duplicate points."""
    N, d = 3000, 5
    X = np.floor(W.uniform(77, (N, d)) * 4.0).astype(dtype)
    X2 = W.sq_norms(X)
    alpha = W.permutation(78, N)[:2500].astype(np.int32)
    beta = W.permutation(79, N)[:700].astype(np.int32)
    for k in (1, 7, 32, 64, 150):
        D, I = run_var1(X, X2, alpha, beta, k)
        big = 1.79e308 if dtype == np.float64 else 1.79e30
        Din = np.full((beta.size, k), big, dtype=dtype)
        Iin = np.full((beta.size, k), -1, dtype=np.int32)
        check_against_oracle(oracle, X, X2, alpha, beta, k, D, I, Din, Iin, exact_float=True)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_merge_sequence_and_duplicates(oracle, dtype):
    """Three calls into the same heaps: disjoint candidates, then a set overlapping both the
    earlier candidates (duplicate entries) and the queries themselves (zero distances)."""
    N, d, k = 6000, 24, 20
    X = W.uniform_table(55, N, d, dtype)
    X2 = W.sq_norms(X)
    beta = W.permutation(56, N)[:500].astype(np.int32)
    sets = [W.permutation(57, N)[:1500], W.permutation(58, N)[:1500],
            np.concatenate([W.permutation(57, N)[:300], beta[:200]])]
    big = 1.79e308 if dtype == np.float64 else 1.79e30
    D = np.full((beta.size, k), big, dtype=dtype)
    I = np.full((beta.size, k), -1, dtype=np.int32)
    for s in sets:
        alpha = np.ascontiguousarray(s, dtype=np.int32)
        Din, Iin = D.copy(), I.copy()
        D, I = run_var1(X, X2, alpha, beta, k, Din, Iin)
        check_against_oracle(oracle, X, X2, alpha, beta, k, D, I, Din, Iin)


def test_infinite_sentinels_and_fewer_candidates(oracle):
    """Heaps initialised with +inf (not 1.79e308) and fewer candidates than k."""
    N, d, k = 400, 6, 40
    X = W.uniform_table(61, N, d)
    X2 = W.sq_norms(X)
    alpha = W.permutation(62, N)[:25].astype(np.int32)
    beta = W.permutation(63, N)[:90].astype(np.int32)
    Din = np.full((90, k), np.inf)
    Iin = np.full((90, k), -1, dtype=np.int32)
    D, I = run_var1(X, X2, alpha, beta, k, Din, Iin)
    assert np.all((I >= 0).sum(axis=1) == 25)
    check_against_oracle(oracle, X, X2, alpha, beta, k, D, I, Din, Iin)


def test_config2_sampled_rows_device_api(oracle):
    """Config 2 at full size through the device entry point (N=1,048,576, d=64, 65,536 queries,
    262,144 references, k=32, FP32); 384 sampled rows checked against the FP64 oracle."""
    import torch
    p = W.config2()
    dev = torch.device("cuda:0")
    X = torch.from_numpy(p.X).to(dev)
    X2 = torch.from_numpy(p.X2).to(dev)
    alpha = torch.from_numpy(p.alpha).to(dev)
    beta = torch.from_numpy(p.beta).to(dev)
    D = torch.full((p.n, p.k), float("inf"), device=dev)
    I = torch.full((p.n, p.k), -1, dtype=torch.int32, device=dev)
    G.knn_device(X, X2, alpha, X, X2, beta, D, I)
    Dh, Ih = D.cpu().numpy(), I.cpu().numpy()
    assert is_maxheap(Dh)
    rows = W.permutation(5, p.n)[:384]
    sub_beta = np.ascontiguousarray(p.beta[rows])
    check_against_oracle(oracle, p.X, p.X2, p.alpha, sub_beta, p.k, Dh[rows], Ih[rows],
                         np.full((384, p.k), np.inf, dtype=np.float32),
                         np.full((384, p.k), -1, dtype=np.int32))


def test_device_index_out_of_range_is_reported():
    """An index outside the table is caught by the gather (never read) and reported."""
    import torch
    dev = torch.device("cuda:0")
    X = torch.rand(100, 8, device=dev)
    X2 = (X * X).sum(1)
    alpha = torch.arange(50, dtype=torch.int32, device=dev)
    alpha[7] = 100  # one past the end
    beta = torch.arange(50, 60, dtype=torch.int32, device=dev)
    D = torch.full((10, 4), float("inf"), device=dev)
    I = torch.full((10, 4), -1, dtype=torch.int32, device=dev)
    with pytest.raises(G.GsknnError):
        G.knn_device(X, X2, alpha, X, X2, beta, D, I)
    # the library stays usable afterwards
    alpha[7] = 7
    G.knn_device(X, X2, alpha, X, X2, beta, D, I)
