"""GPU tests of the tensor-core pass's threshold machinery and its variants.

1. Partition bound: every epilogue part keeps a heap of ceil(k/2) entries, publishes its root,
   and a row thresholds on the second smallest root it can see, its own CTA's two parts and
   the roots of up to three other splits. Cases here stress its edges: odd k and k = 1 (heaps of
   ceil(k/2)); few queries against many candidates, so the plan takes many splits and a row reads
   only a window of four of them.
2. Norm column: where it fits, the candidate norms enter through the MMA (split BF16, BF16 from
   d = 128). Turning it off (GSKNN_TC_FOLD=0, read at plan time) must give identical results,
   since both forms end in the exact FP64 re-rank.
3. The BF16 re-rank holds the band above the approximate k-th back (k <= 64), filters it against
   the exact k-th + E, and bounds it by the incoming heap row: merges into existing heaps.

Parity is against the FP64 oracle (`dgsknn_ref` semantics on the float inputs upcast, the
caller's norms, ties to the lower index), as in test_gpu_tc.py.
"""
import numpy as np
import pytest

from knn_check import is_maxheap
from rnn_b200 import workloads as W
from test_gpu_tc import _run, assert_close, assert_same_sets

pytestmark = pytest.mark.gpu


def _problem(seed, N, d, m, n):
    X = W.gaussian_mixture_table(seed, N, d, dtype=np.float32)
    X2 = W.sq_norms(X)
    alpha = W.permutation(seed + 1, N)[:m].astype(np.int32)
    beta = W.permutation(seed + 2, N)[:n].astype(np.int32)
    return X, X2, alpha, beta


def _check(oracle, X, X2, alpha, beta, k, D, I, Din=None, Iin=None):
    n = beta.size
    if Din is None:
        Din = np.full((n, k), np.inf, dtype=np.float32)
        Iin = np.full((n, k), -1, dtype=np.int32)
    De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta, Din, Iin, clamp=True)
    assert is_maxheap(D)
    assert_same_sets(X, X2, beta, I, Ie, De)
    assert_close(np.sort(D.astype(np.float64), axis=1), De)


@pytest.mark.parametrize("mode", ["tf32", "bf16", "bf16x3"])
@pytest.mark.parametrize("k", [1, 33])
def test_odd_and_single_k(oracle, mode, k):
    X, X2, alpha, beta = _problem(1100 + k, 9000, 64, 8000, 700)
    D, I, _, _ = _run(mode, X, X2, alpha, beta, k, want_C=False)
    _check(oracle, X, X2, alpha, beta, k, D, I)


@pytest.mark.parametrize("mode", ["tf32", "bf16", "bf16x3"])
def test_many_splits_window(oracle, mode):
    """200 queries (2 query tiles) against 60,000 candidates: the plan spreads each query tile
    over many candidate splits, and each row reads the roots of a window of four of them."""
    X, X2, alpha, beta = _problem(1200, 61000, 32, 60000, 200)
    D, I, _, _ = _run(mode, X, X2, alpha, beta, 48, want_C=False)
    _check(oracle, X, X2, alpha, beta, 48, D, I)


@pytest.mark.parametrize("mode,d", [("bf16x3", 64), ("bf16", 128), ("bf16", 256)])
def test_norm_column_on_and_off_identical(monkeypatch, mode, d):
    X, X2, alpha, beta = _problem(1300 + d, 12000, d, 10000, 900)
    D1, I1, C1, m1 = _run(mode, X, X2, alpha, beta, 32)
    monkeypatch.setenv("GSKNN_TC_FOLD", "0")
    D0, I0, C0, m0 = _run(mode, X, X2, alpha, beta, 32)
    monkeypatch.delenv("GSKNN_TC_FOLD")
    assert np.array_equal(I1, I0)
    assert np.array_equal(D1, D0)
    # both approximate blocks within their own bound E of the FP64 distances
    Q = X[beta].astype(np.float64)
    Cm = X[alpha].astype(np.float64)
    exact = -2.0 * Q @ Cm.T + X2[alpha].astype(np.float64)[None, :] \
        + X2[beta].astype(np.float64)[:, None]
    for C, mg in ((C1, m1), (C0, m0)):
        assert np.all(np.isfinite(C))
        assert np.all(np.abs(C.astype(np.float64) - exact) <= (mg.astype(np.float64) / 2)[:, None])


@pytest.mark.parametrize("k", [16, 64])
def test_bf16_held_band_merges_into_existing_heaps(oracle, k):
    """BF16 (the held-band re-rank) merging a second candidate set into the first call's heaps:
    the incoming rows bound the band from the start."""
    X, X2, _, beta = _problem(1400 + k, 14000, 128, 1, 600)
    a1 = W.permutation(1411, 14000)[:5000].astype(np.int32)
    a2 = np.concatenate([W.permutation(1412, 14000)[:6000], beta[:40]]).astype(np.int32)
    D1, I1, _, _ = _run("bf16", X, X2, a1, beta, k, want_C=False)
    D2, I2, _, _ = _run("bf16", X, X2, a2, beta, k, D=D1.copy(), I=I1.copy(), want_C=False)
    _check(oracle, X, X2, a2, beta, k, D2, I2, D1, I1)

