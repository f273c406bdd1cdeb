"""CPU tests of the batching form's host side: the randomized-tree leaf builder and the
oracle's restatement of the all-nearest-neighbour semantics."""
import numpy as np
import pytest

from rnn_b200 import batch as B
from rnn_b200 import workloads as W


def _check_partition(lv, N, ntrees, lmin, lmax):
    assert lv.ptr[0] == 0 and lv.ptr[-1] == ntrees * N
    assert np.all(np.diff(lv.ptr) > 0)
    for t in range(ntrees):
        sel = np.nonzero(lv.tree == t)[0]
        assert sel.size > 0
        pts = np.concatenate([lv.pts[lv.ptr[l]:lv.ptr[l + 1]] for l in sel])
        assert np.array_equal(np.sort(pts), np.arange(N)), f"tree {t} is not a partition"
        sizes = np.diff(lv.ptr)[sel]
        if N >= lmin:
            assert sizes.min() >= lmin and sizes.max() <= lmax


@pytest.mark.parametrize("N,lmin,lmax", [(10000, 64, 256), (5000, 100, 300), (50, 64, 256),
                                         (257, 64, 128)])
def test_rkdt_leaves_partition_each_tree(N, lmin, lmax):
    X = W.gaussian_mixture_table(31, N, 12, dtype=np.float32)
    lv = B.rkdt_leaves(X, 5, lmin, lmax, seed=7)
    _check_partition(lv, N, 5, lmin, lmax)


def test_rkdt_leaves_deterministic_and_seeded():
    X = W.gaussian_mixture_table(32, 8000, 16, dtype=np.float32)
    a = B.rkdt_leaves(X, 4, 64, 256, seed=11, threads=1)
    b = B.rkdt_leaves(X, 4, 64, 256, seed=11, threads=4)
    c = B.rkdt_leaves(X, 4, 64, 256, seed=12)
    assert np.array_equal(a.ptr, b.ptr) and np.array_equal(a.pts, b.pts)
    assert not np.array_equal(a.pts, c.pts)
    # trees of one build differ from each other
    t0 = a.pts[:8000]
    t1 = a.pts[8000:16000]
    assert not np.array_equal(t0, t1)


def test_rkdt_leaves_are_spatially_local():
    """Projection splits put near points together: leaves are far tighter than the whole set,
    and a point's true nearest neighbours share its leaf far more often than chance."""
    N, d = 6000, 16
    X = W.gaussian_mixture_table(33, N, d, dtype=np.float32).astype(np.float64)
    lv = B.rkdt_leaves(X.astype(np.float32), 1, 64, 256, seed=3)
    intra = []
    leaf_of = np.empty(N, dtype=np.int64)
    for l in range(lv.nleaves):
        p = lv.pts[lv.ptr[l]:lv.ptr[l + 1]]
        leaf_of[p] = l
        c = X[p].mean(0)
        intra.append(((X[p] - c) ** 2).sum(1).mean())
    glob = ((X - X.mean(0)) ** 2).sum(1).mean()
    assert np.mean(intra) < 0.4 * glob
    Dm = ((X[:400, None, :] - X[None, :, :]) ** 2).sum(-1)
    nn = np.argsort(Dm, axis=1)[:, 1:11]
    recall = (leaf_of[nn] == leaf_of[:400, None]).mean()
    assert recall > 10.0 / lv.nleaves  # a random partition gives about 1 / nleaves


def test_rkdt_leaves_rejects_bad_bounds():
    X = np.zeros((100, 4), np.float32)
    with pytest.raises(Exception):
        B.rkdt_leaves(X, 1, 64, 100, seed=0)  # leaf_max < 2 leaf_min


def test_allnn_oracle_matches_exact_selection_on_one_leaf(oracle):
    """With a single leaf holding every point the all-NN oracle is the exact kNN oracle."""
    N, d, k = 700, 9, 12
    X = W.gaussian_mixture_table(34, N, d, dtype=np.float32)
    X2 = W.sq_norms(X)
    ptr = np.array([0, N], np.int32)
    pts = W.permutation(35, N).astype(np.int32)
    Da, Ia = oracle.allnn_leaves(k, X, X2, ptr, pts)
    allp = np.arange(N, dtype=np.int32)
    De, Ie = oracle.knn_exact(k, X, X2, allp, X, X2, allp)
    assert np.array_equal(Ia, Ie)
    assert np.array_equal(Da, De)


def test_allnn_oracle_deduplicates_across_leaves(oracle):
    """The same leaf listed twice (two trees that agree) gives the same result as once."""
    N, d, k = 400, 5, 10
    X = W.uniform_table(36, N, d).astype(np.float32)
    X2 = W.sq_norms(X)
    lv = B.rkdt_leaves(X, 1, 32, 64, seed=5)
    ptr2 = np.concatenate([lv.ptr, lv.ptr[1:] + lv.ptr[-1]]).astype(np.int32)
    pts2 = np.concatenate([lv.pts, lv.pts]).astype(np.int32)
    D1, I1 = oracle.allnn_leaves(k, X, X2, lv.ptr, lv.pts)
    D2, I2 = oracle.allnn_leaves(k, X, X2, ptr2, pts2)
    assert np.array_equal(I1, I2) and np.array_equal(D1, D2)
    for row in I1:
        real = row[row >= 0]
        assert np.unique(real).size == real.size


def test_point_table_round_trip(tmp_path):
    """The on-disk table: rows and norms back bit for bit through the read-only mapping; norms
    computed in double when not given."""
    X = W.gaussian_mixture_table(33, 3001, 7, dtype=np.float32)
    X2 = W.sq_norms(X).astype(np.float32)
    p1, p2 = str(tmp_path / "a.tbl"), str(tmp_path / "b.tbl")
    B.write_table(p1, X, X2)
    B.write_table(p2, X)
    t1, t2 = B.Table(p1), B.Table(p2)
    assert (t1.N, t1.d) == (3001, 7)
    assert np.array_equal(t1.X, X) and np.array_equal(t1.X2, X2)
    assert np.array_equal(t2.X2, X2)  # FP64 sums rounded to float, as sq_norms
    with open(p1, "rb") as f:
        head = f.read(64)
    assert head[:8] == b"GSKNNTB1"
    assert int.from_bytes(head[16:24], "little") == 3001
    assert (tmp_path / "a.tbl").stat().st_size == 64 + 3001 * 8 * 4
    t1.close()
    t2.close()


def test_point_table_rejects_other_files(tmp_path):
    from rnn_b200 import gsknn as G
    bad = tmp_path / "bad.tbl"
    bad.write_bytes(b"NOTATABLE" + bytes(100))
    with pytest.raises(G.GsknnError):
        B.Table(str(bad))
    short = tmp_path / "short.tbl"
    X = np.ones((10, 4), np.float32)
    B.write_table(str(short), X)
    data = short.read_bytes()
    short.write_bytes(data[:-8])  # truncated norms
    with pytest.raises(G.GsknnError):
        B.Table(str(short))
    with pytest.raises(G.GsknnError):
        B.Table(str(tmp_path / "missing.tbl"))
