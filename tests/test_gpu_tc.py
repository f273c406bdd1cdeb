"""GPU tests of the tensor-core precision form (TF32, BF16, split BF16 + FP64 re-rank).

1. The approximate distance block the tcgen05 pass computes lies within the stated bound E of
   the FP64 distance for every pair (checks the MMA/TMA/TMEM data path and the error bound).
2. After the FP64 re-rank the neighbour sets are exactly the FP64 oracle's (ties to the lower
   index) and distances match the FP64 values to float rounding.
"""
import ctypes

import numpy as np
import pytest

from knn_check import is_maxheap, sorted_rows
from rnn_b200 import gsknn as G
from rnn_b200 import workloads as W

pytestmark = pytest.mark.gpu

MODES = {"tf32": 2, "bf16": 3, "bf16x3": 4}


def _bind():
    L = G.lib()
    f = L.gsknn_tc_distances
    vp, ci, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
    f.argtypes = [ci, ci, ci, ci, ci, vp, vp, ll, vp, vp, vp, ll, vp, vp, vp, ci, vp, ll, vp, vp]
    f.restype = ci
    return f


def _run(mode, X, X2, alpha, beta, k, D=None, I=None, want_C=True):
    import torch
    dev = torch.device("cuda:0")
    f = _bind()
    Xd = torch.from_numpy(X).to(dev)
    X2d = torch.from_numpy(X2).to(dev)
    a = torch.from_numpy(alpha).to(dev)
    b = torch.from_numpy(beta).to(dev)
    n, m = beta.size, alpha.size
    if D is None:
        Dd = torch.full((n, k), float("inf"), device=dev)
        Id = torch.full((n, k), -1, dtype=torch.int32, device=dev)
    else:
        Dd = torch.from_numpy(D).to(dev)
        Id = torch.from_numpy(I).to(dev)
    C = torch.full((n, m), float("nan"), device=dev) if want_C else None
    margin = torch.zeros(n, device=dev)
    st = torch.cuda.current_stream(dev)
    rc = f(MODES[mode], m, n, X.shape[1], k, Xd.data_ptr(), X2d.data_ptr(), X.shape[0],
           a.data_ptr(), Xd.data_ptr(), X2d.data_ptr(), X.shape[0], b.data_ptr(), Dd.data_ptr(),
           Id.data_ptr(), k, C.data_ptr() if C is not None else None, m, margin.data_ptr(),
           st.cuda_stream)
    assert rc == 0, G.last_error()
    assert G.lib().gsknn_stream_status(ctypes.c_void_p(st.cuda_stream)) == 0, G.last_error()
    return (Dd.cpu().numpy(), Id.cpu().numpy(), None if C is None else C.cpu().numpy(),
            margin.cpu().numpy())


def _exact_block(X, X2, alpha, beta):
    Q = X[beta].astype(np.float64)
    C = X[alpha].astype(np.float64)
    return np.maximum(0.0, -2.0 * Q @ C.T + X2[alpha].astype(np.float64)[None, :]
                      + X2[beta].astype(np.float64)[:, None])


@pytest.mark.parametrize("mode", ["tf32", "bf16", "bf16x3"])
@pytest.mark.parametrize("d", [64, 100, 256])
def test_tc_distance_block_within_bound(mode, d):
    N, m, n, k = 3000, 1100, 300, 16
    X = W.gaussian_mixture_table(400 + d, N, d, dtype=np.float32)
    X2 = W.sq_norms(X)
    alpha = W.permutation(401, N)[:m].astype(np.int32)
    beta = W.permutation(402, N)[:n].astype(np.int32)
    D, I, C, margin = _run(mode, X, X2, alpha, beta, k)
    ex = _exact_block(X, X2, alpha, beta)
    # d' is unclamped: compare with the unclamped exact value
    exu = -2.0 * X[beta].astype(np.float64) @ X[alpha].astype(np.float64).T \
        + X2[alpha].astype(np.float64)[None, :] + X2[beta].astype(np.float64)[:, None]
    assert np.all(np.isfinite(C))
    E = margin / 2.0
    err = np.abs(C.astype(np.float64) - exu)
    assert np.all(err <= E[:, None]), f"max err/E = {np.max(err / E[:, None]):.3f}"
    # the bound should not be absurdly loose either (at most ~1000x the observed error)
    assert np.median(E) < 1e3 * max(np.max(err), 1e-12)
    del ex


@pytest.mark.parametrize("mode", ["tf32", "bf16", "bf16x3"])
@pytest.mark.parametrize("shape", [(2000, 300, 64, 32), (5000, 257, 256, 64), (700, 33, 100, 16),
                                   (3000, 129, 40, 100), (50, 20, 16, 64)])
def test_tc_knn_exact_sets(oracle, mode, shape):
    m, n, d, k = shape
    N = m + n + 11
    X = W.gaussian_mixture_table(500 + d + m, N, d, dtype=np.float32)
    X2 = W.sq_norms(X)
    alpha = W.permutation(501 + m, N)[:m].astype(np.int32)
    beta = W.permutation(502 + n, N)[:n].astype(np.int32)
    D, I, _, _ = _run(mode, X, X2, alpha, beta, k, want_C=False)
    assert is_maxheap(D)
    Din = np.full((n, k), np.inf, dtype=np.float32)
    Iin = np.full((n, k), -1, dtype=np.int32)
    De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta, Din, Iin, clamp=True)
    assert_same_sets(X, X2, beta, I, Ie, De)
    assert_close(np.sort(D.astype(np.float64), axis=1), De)


def assert_close(Ds, De, rel=1e-6, abs_=1e-9):
    """Re-ranked distances are FP64 values rounded to float: within float rounding, plus an
    absolute allowance for FP64 cancellation in -2<q,c> + |c|^2 + |q|^2 near zero."""
    fin = np.isfinite(De)
    err = np.abs(Ds[fin] - De[fin])
    tol = rel * np.abs(De[fin]) + abs_
    if not np.all(err <= tol):
        i = int(np.argmax(err - tol))
        raise AssertionError(f"distance mismatch: got {Ds[fin][i]!r} want {De[fin][i]!r}")


def assert_same_sets(X, X2, beta, I, Ie, De):
    """Index sets equal row by row; on failure report the FP64 distances involved."""
    bad = [j for j in range(I.shape[0]) if not np.array_equal(np.sort(I[j]), np.sort(Ie[j]))]
    if bad:
        from knn_check import exact_dists
        j = bad[0]
        extra = np.setdiff1d(I[j], Ie[j])
        missing = np.setdiff1d(Ie[j], I[j])
        de = exact_dists(X, beta[j], extra[extra >= 0], X2) if extra.size else []
        dm = exact_dists(X, beta[j], missing[missing >= 0], X2) if missing.size else []
        raise AssertionError(f"{len(bad)} rows differ; row {j}: kth={De[j].max()!r} "
                             f"extra={list(zip(extra, de))} missing={list(zip(missing, dm))}")


@pytest.mark.parametrize("mode", ["tf32", "bf16x3"])
def test_tc_merge_into_existing_heaps(oracle, mode):
    """Second call merges a fresh candidate set into the heaps of the first (in place)."""
    N, d, k = 6000, 128, 24
    X = W.gaussian_mixture_table(600, N, d, dtype=np.float32)
    X2 = W.sq_norms(X)
    beta = W.permutation(601, N)[:400].astype(np.int32)
    a1 = W.permutation(602, N)[:2500].astype(np.int32)
    a2 = np.concatenate([W.permutation(603, N)[:2000], beta[:50]]).astype(np.int32)
    D1, I1, _, _ = _run(mode, X, X2, a1, beta, k, want_C=False)
    D2, I2, _, _ = _run(mode, X, X2, a2, beta, k, D=D1.copy(), I=I1.copy(), want_C=False)
    De, Ie = oracle.knn_exact(k, X, X2, a2, X, X2, beta, D1, I1, clamp=True)
    assert_same_sets(X, X2, beta, I2, Ie, De)
    assert is_maxheap(D2)


def test_tc_ties_and_duplicates_exact(oracle):
    """Integer coordinates: many exact ties; the re-rank resolves them by the lower index."""
    N, d, k = 2500, 8, 20
    X = np.floor(W.uniform(700, (N, d)) * 4.0).astype(np.float32)
    X2 = W.sq_norms(X)
    alpha = W.permutation(701, N)[:2000].astype(np.int32)
    beta = W.permutation(702, N)[:300].astype(np.int32)
    for mode in ("tf32", "bf16", "bf16x3"):
        D, I, _, _ = _run(mode, X, X2, alpha, beta, k, want_C=False)
        De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta,
                                  np.full((300, k), np.inf, dtype=np.float32),
                                  np.full((300, k), -1, dtype=np.int32), clamp=True)
        Ds, Is = sorted_rows(D.astype(np.float64), I)
        assert np.array_equal(Is, Ie), mode
        assert np.array_equal(Ds, De), mode


def _traced_run(mode, X, X2, alpha, beta, k):
    """_run with the library's launch tracer on; returns (D, I, kernel brackets seen)."""
    import json
    L = G.lib()
    buf = ctypes.create_string_buffer(1 << 16)
    L.gsknn_trace_read(buf, len(buf))
    L.gsknn_trace_enable(1)
    try:
        D, I, _, _ = _run(mode, X, X2, alpha, beta, k, want_C=False)
    finally:
        L.gsknn_trace_enable(0)
    L.gsknn_trace_read(buf, len(buf))
    return D, I, json.loads(buf.value.decode() or "{}")


def test_bf16_log_overflow_escalates_to_split_bf16(oracle):
    """Clustered data at d = 64: the BF16 band holds most of a query's cluster, its logs
    overflow, and those queries run again in split BF16 (the escalation pass) instead of the
    FP64 brute force. Results stay the exact FP64 sets."""
    N, d, k = 40000, 64, 32
    X = W.gaussian_mixture_table(801, N, d, dtype=np.float32)
    X2 = W.sq_norms(X)
    alpha = W.permutation(802, N)[:30000].astype(np.int32)
    beta = W.permutation(803, N)[:1000].astype(np.int32)
    D, I, tr = _traced_run("bf16", X, X2, alpha, beta, k)
    assert "tc_escalate" in tr, tr  # the escalation pass is launched (its work is on-device)
    De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta,
                              np.full((1000, k), np.inf, dtype=np.float32),
                              np.full((1000, k), -1, dtype=np.int32), clamp=True)
    assert_same_sets(X, X2, beta, I, Ie, De)
    assert_close(np.sort(D.astype(np.float64), axis=1), De)
    assert is_maxheap(D)


@pytest.mark.parametrize("mode", ["tf32", "bf16", "bf16x3"])
def test_all_equal_points_go_to_brute_force(oracle, mode):
    """Every candidate at the same distance: every band overflows in every format, so the
    queries end in the FP64 brute force, which keeps the lowest ids (the tie rule)."""
    N, d, k = 3000, 32, 16
    X = np.tile(W.uniform(804, (1, d)).astype(np.float32), (N, 1))
    X[:5] += 1.0  # a few distinct points, far away
    X2 = W.sq_norms(X)
    alpha = W.permutation(805, N)[:2500].astype(np.int32)
    beta = W.permutation(806, N)[:200].astype(np.int32)
    D, I, _ = _traced_run(mode, X, X2, alpha, beta, k)
    De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta,
                              np.full((200, k), np.inf, dtype=np.float32),
                              np.full((200, k), -1, dtype=np.int32), clamp=True)
    Ds, Is = sorted_rows(D.astype(np.float64), I)
    assert np.array_equal(Is, Ie)
