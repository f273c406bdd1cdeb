"""GPU tests of the batching form (all-nearest-neighbour over randomized-tree leaves, one
persistent graph-replayed launch per pass, heaps merged across passes without duplicates).

Parity is against the oracle's restatement (oracle_allnn_leaves_s): per point, the k nearest
among the union of its leaf-mates and its incoming heap row, FP64 distances, lower id first.
On small-integer coordinates FP32 arithmetic is exact, so rows must match exactly (tie rule
included); on general data every distance lies within FP32 rounding of the FP64 value and sets
agree outside that band.
"""
import numpy as np
import pytest

from knn_check import compare_sets, exact_dists, is_maxheap, sorted_rows
from rnn_b200 import batch as B
from rnn_b200 import gsknn as G
from rnn_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dev(*arrays):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]


def _heap(N, k, D0=None, I0=None):
    import torch
    if D0 is None:
        D = torch.full((N, k), float("inf"), device="cuda")
        I = torch.full((N, k), -1, dtype=torch.int32, device="cuda")
    else:
        D, I = _dev(D0, I0)
    return D, I


def _int_table(seed, N, d):
    return np.floor(W.uniform(seed, (N, d)) * 4.0).astype(np.float32)


def _leaves_concat(lvs):
    ptr, pts = [0], []
    for lv in lvs:
        for l in range(lv.nleaves):
            seg = lv.pts[lv.ptr[l]:lv.ptr[l + 1]]
            pts.append(seg)
            ptr.append(ptr[-1] + seg.size)
    return np.asarray(ptr, np.int32), np.concatenate(pts).astype(np.int32)


def _run(X, X2, k, passes, shape, T, leaf_min, D0=None, I0=None):
    N = X.shape[0]
    Xd, X2d = _dev(X, X2)
    D, I = _heap(N, k, D0, I0)
    job = B.BatchJob(Xd, X2d, D, I, k, trees_per_pass=T, leaf_min=leaf_min, shape=shape)
    for lv in passes:
        job.run_pass(lv)
    job.sync()
    info = job.info()
    job.close()
    return D.cpu().numpy(), I.cpu().numpy(), info


def _assert_unique_rows(I):
    for row in I:
        real = row[row >= 0]
        assert np.unique(real).size == real.size


@pytest.mark.parametrize("shape", [0, 1, 2, 3])
def test_batch_exact_integer_data_every_shape(oracle, shape):
    N, d, k, T = 5000, 8, 16, 3
    X = _int_table(900, N, d)
    X2 = W.sq_norms(X)
    lv = B.rkdt_leaves(X, 2 * T, 64, 256, seed=901)
    passes = [lv.select_trees(range(0, T)), lv.select_trees(range(T, 2 * T))]
    D, I, info = _run(X, X2, k, passes, shape, T, 64)
    assert info["shape"] == shape
    assert is_maxheap(D)
    _assert_unique_rows(I)
    ptr, pts = _leaves_concat(passes)
    De, Ie = oracle.allnn_leaves(k, X, X2, ptr, pts)
    Ds, Is = sorted_rows(D.astype(np.float64), I)
    assert np.array_equal(Is, Ie)
    assert np.array_equal(Ds, De)


def test_batch_autotuned_gaussian_mixture(oracle):
    N, d, k, T = 20000, 32, 32, 4
    X = W.gaussian_mixture_table(910, N, d, dtype=np.float32)
    X2 = W.sq_norms(X)
    lv = B.rkdt_leaves(X, 2 * T, 100, 400, seed=911)
    passes = [lv.select_trees(range(0, T)), lv.select_trees(range(T, 2 * T))]
    B.forget_tuning()
    D, I, info = _run(X, X2, k, passes, -1, T, 100)
    assert info["shape"] in (0, 1, 2, 3)
    assert len(info["tune_ms"]) == 4 and min(info["tune_ms"].values()) > 0
    assert is_maxheap(D)
    _assert_unique_rows(I)
    ptr, pts = _leaves_concat(passes)
    De, Ie = oracle.allnn_leaves(k, X, X2, ptr, pts)
    band = 4e-6 * np.maximum(1.0, np.abs(De).max(axis=1)) * 16
    eq, bad = compare_sets(I, Ie, De, band, dist_of=lambda j, ids: exact_dists(X, j, ids, X2))
    assert not bad, bad[:5]
    # every returned distance is the FP32 rounding of its id's FP64 distance
    for j in range(0, N, 997):
        ids = I[j][I[j] >= 0]
        de = exact_dists(X, j, ids, X2)
        assert np.all(np.abs(D[j][I[j] >= 0] - de) <= 4e-6 * np.maximum(1.0, de) * 16)


def test_batch_partial_trees_tiny_leaves_and_k_above_leaf(oracle):
    """Hand-made leaves: sizes 1, 3, 63, 64, 65, 200; tree 1 covers only part of the points;
    k = 40 exceeds several leaves, so those heaps keep +inf / -1 sentinels."""
    N, d, k = 600, 6, 40
    X = _int_table(920, N, d)
    X2 = W.sq_norms(X)
    perm = W.permutation(921, N).astype(np.int32)
    sizes0 = [1, 3, 63, 64, 65, 200, 204]          # tree 0: all 600 points
    sizes1 = [50, 130, 7]                          # tree 1: 187 points only
    ptr, tree, pts = [0], [], []
    off = 0
    for s in sizes0:
        pts.append(perm[off:off + s]); off += s; ptr.append(ptr[-1] + s); tree.append(0)
    perm1 = W.permutation(922, N).astype(np.int32)
    off = 0
    for s in sizes1:
        pts.append(perm1[off:off + s]); off += s; ptr.append(ptr[-1] + s); tree.append(1)
    lv = B.Leaves(np.asarray(ptr, np.int32), np.concatenate(pts), np.asarray(tree, np.int32))
    for shape in (0, 1, 3):
        D, I, _ = _run(X, X2, k, [lv], shape, 2, 1)
        assert is_maxheap(D)
        _assert_unique_rows(I)
        De, Ie = oracle.allnn_leaves(k, X, X2, lv.ptr, lv.pts)
        Ds, Is = sorted_rows(D.astype(np.float64), I)
        assert np.array_equal(Is, Ie), shape
        assert np.array_equal(Ds[np.isfinite(De)], De[np.isfinite(De)])
        assert np.all(np.isinf(Ds[~np.isfinite(De)]))


@pytest.mark.parametrize("shape", [1, 3])
def test_batch_graph_replays_many_passes(oracle, shape):
    """Four passes (for the CUDA-core shape through one captured graph; for the tensor-core
    shape tree by tree, each re-rank merging into the heap without entering an id twice),
    checked after every pass."""
    import torch
    N, d, k, T = 8000, 10, 24, 2
    X = _int_table(930, N, d)
    X2 = W.sq_norms(X)
    lv = B.rkdt_leaves(X, 4 * T, 80, 320, seed=931)
    Xd, X2d = _dev(X, X2)
    D, I = _heap(N, k)
    job = B.BatchJob(Xd, X2d, D, I, k, trees_per_pass=T, leaf_min=80, shape=shape)
    done = []
    for p in range(4):
        lp = lv.select_trees(range(p * T, (p + 1) * T))
        job.run_pass(lp)
        job.sync()
        done.append(lp)
        ptr, pts = _leaves_concat(done)
        De, Ie = oracle.allnn_leaves(k, X, X2, ptr, pts)
        Ds, Is = sorted_rows(D.cpu().numpy().astype(np.float64), I.cpu().numpy())
        assert np.array_equal(Is, Ie), f"pass {p}"
        assert np.array_equal(Ds, De), f"pass {p}"
    job.close()
    torch.cuda.synchronize()


@pytest.mark.parametrize("shape", [0, 3])
def test_batch_merges_into_an_existing_heap(oracle, shape):
    """Heaps first filled by sgsknn (FP32 mode, random candidates), then refined by two passes."""
    N, d, k, T = 4000, 8, 16, 2
    X = _int_table(940, N, d)
    X2 = W.sq_norms(X)
    alpha = W.permutation(941, N)[:500].astype(np.int32)
    beta = np.arange(N, dtype=np.int32)
    D0 = np.full((N, k), np.inf, dtype=np.float32)
    I0 = np.full((N, k), -1, dtype=np.int32)
    prev = G.get_mode()
    G.set_mode(G.MODE_FP32)
    try:
        G.sgsknn(d, k, X, X2, beta, X, X2, alpha, D0, I0)
    finally:
        G.set_mode(prev)
    lv = B.rkdt_leaves(X, 2 * T, 64, 256, seed=942)
    passes = [lv.select_trees(range(0, T)), lv.select_trees(range(T, 2 * T))]
    D, I, _ = _run(X, X2, k, passes, shape, T, 64, D0, I0)
    _assert_unique_rows(I)
    ptr, pts = _leaves_concat(passes)
    De, Ie = oracle.allnn_leaves(k, X, X2, ptr, pts, D0, I0)
    Ds, Is = sorted_rows(D.astype(np.float64), I)
    assert np.array_equal(Is, Ie)
    assert np.array_equal(Ds, De)


@pytest.mark.parametrize("shape", [1, 3])
def test_batch_reports_a_point_outside_the_table(shape):
    N, d, k = 1000, 4, 8
    X = _int_table(950, N, d)
    X2 = W.sq_norms(X)
    pts = np.arange(N, dtype=np.int32)
    pts[17] = N  # one past the end: packed as padding, reported, never read
    lv = B.Leaves(np.array([0, 500, N], np.int32), pts, np.array([0, 0], np.int32))
    Xd, X2d = _dev(X, X2)
    D, I = _heap(N, k)
    job = B.BatchJob(Xd, X2d, D, I, k, trees_per_pass=1, leaf_min=100, shape=shape)
    job.run_pass(lv)
    with pytest.raises(G.GsknnError):
        job.sync()
    job.close()


def test_batch_tensor_core_shape_gaussian_mixture(oracle):
    """The tensor-core shape on clustered data (d = 64, k = 32, leaves of 256..2048 points, two
    passes of four trees): exact FP64 neighbour sets, distances the FP64 values in float."""
    N, d, k, T = 30000, 64, 32, 4
    X = W.gaussian_mixture_table(960, N, d, dtype=np.float32)
    X2 = W.sq_norms(X)
    lv = B.rkdt_leaves(X, 2 * T, 256, 2048, seed=961)
    passes = [lv.select_trees(range(0, T)), lv.select_trees(range(T, 2 * T))]
    D, I, info = _run(X, X2, k, passes, 3, T, 256)
    assert info["shape"] == 3
    assert is_maxheap(D)
    _assert_unique_rows(I)
    ptr, pts = _leaves_concat(passes)
    De, Ie = oracle.allnn_leaves(k, X, X2, ptr, pts)
    bad = [j for j in range(N) if not np.array_equal(np.sort(I[j]), np.sort(Ie[j]))]
    assert not bad, bad[:5]
    Ds = np.sort(D.astype(np.float64), axis=1)
    assert np.all(np.abs(Ds - De) <= 1e-6 * np.abs(De) + 1e-9)
