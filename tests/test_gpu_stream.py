"""GPU tests of the streaming form: the batching form with the point table and the heaps in
host memory (or a table mapped from disk), streamed through a device staging table in groups
of whole leaves.

Bars: the heaps equal a resident batching job's after the same passes, bit for bit (the same
kernels and arithmetic; a point's lists meet in the same merges); on small-integer data the
rows equal the oracle's all-nearest-neighbour restatement exactly, tie rule included.
"""
import numpy as np
import pytest

from knn_check import is_maxheap, sorted_rows
from rnn_b200 import batch as B
from rnn_b200 import gsknn as G
from rnn_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _int_table(seed, N, d):
    return np.floor(W.uniform(seed, (N, d)) * 4.0).astype(np.float32)


def _resident(X, X2, k, passes, T, leaf_min, shape):
    import torch
    N = X.shape[0]
    Xd = torch.from_numpy(X).cuda()
    X2d = torch.from_numpy(X2).cuda()
    D = torch.full((N, k), float("inf"), device="cuda")
    I = torch.full((N, k), -1, dtype=torch.int32, device="cuda")
    job = B.BatchJob(Xd, X2d, D, I, k, trees_per_pass=T, leaf_min=leaf_min, shape=shape)
    for lv in passes:
        job.run_pass(lv)
    job.sync()
    job.close()
    return D.cpu().numpy(), I.cpu().numpy()


def _streamed(X, X2, k, passes, group_points, leaf_min, shape, ldD=None):
    N = X.shape[0]
    ldD = k if ldD is None else ldD
    D = np.full((N, ldD), np.inf, np.float32)
    I = np.full((N, ldD), -1, np.int32)
    job = B.StreamJob(X, X2, D, I, k, group_points=group_points, leaf_min=leaf_min, shape=shape)
    infos = []
    for lv in passes:
        job.run_pass(lv)
        infos.append(job.info())
    job.close()
    return D[:, :k].copy(), I[:, :k].copy(), infos


@pytest.mark.parametrize("shape", [0, 2])
def test_stream_equals_resident_job(shape):
    N, d, k, T = 30000, 24, 16, 3
    X = W.gaussian_mixture_table(950, N, d, dtype=np.float32)
    X2 = W.sq_norms(X).astype(np.float32)
    lv = B.rkdt_leaves(X, 2 * T, 64, 256, seed=951)
    passes = [lv.select_trees(range(0, T)), lv.select_trees(range(T, 2 * T))]
    Dr, Ir = _resident(X, X2, k, passes, T, 64, shape)
    Ds, Is, infos = _streamed(X, X2, k, passes, group_points=4000, leaf_min=64, shape=shape)
    assert all(i["groups"] >= T * (N // 4000) for i in infos)
    assert is_maxheap(Ds)
    assert np.array_equal(Ds, Dr) and np.array_equal(Is, Ir)


def test_stream_from_mapped_table_exact(oracle, tmp_path):
    """A table written to disk and mapped read-only; integer coordinates, rows against the
    oracle; heap rows of stride ldD > k keep their tail."""
    N, d, k, T = 12000, 8, 20, 2
    X = _int_table(960, N, d)
    path = str(tmp_path / "pts.tbl")
    B.write_table(path, X)
    tab = B.Table(path)
    lv = B.rkdt_leaves(X, 2 * T, 80, 320, seed=961)
    passes = [lv.select_trees(range(0, T)), lv.select_trees(range(T, 2 * T))]
    ldD = k + 5
    D = np.full((N, ldD), np.inf, np.float32)
    I = np.full((N, ldD), -1, np.int32)
    D[:, k:] = -3.0
    I[:, k:] = -7
    job = B.StreamJob(tab.X, tab.X2, D, I, k, group_points=2500, leaf_min=80, shape=1)
    for p in passes:
        job.run_pass(p)
    job.close()
    assert np.all(D[:, k:] == -3.0) and np.all(I[:, k:] == -7)
    ptr = [0]
    pts = []
    for p in passes:
        for l in range(p.nleaves):
            seg = p.pts[p.ptr[l]:p.ptr[l + 1]]
            pts.append(seg)
            ptr.append(ptr[-1] + seg.size)
    De, Ie = oracle.allnn_leaves(k, X, tab.X2.copy(), np.asarray(ptr, np.int32),
                                 np.concatenate(pts).astype(np.int32))
    Ds, Is = sorted_rows(D[:, :k].astype(np.float64), I[:, :k])
    assert np.array_equal(Is, Ie) and np.array_equal(Ds, De)
    tab.close()


def test_stream_rejects_leaf_larger_than_group():
    N, d, k = 1000, 4, 8
    X = _int_table(970, N, d)
    X2 = W.sq_norms(X).astype(np.float32)
    D = np.full((N, k), np.inf, np.float32)
    I = np.full((N, k), -1, np.int32)
    job = B.StreamJob(X, X2, D, I, k, group_points=300, leaf_min=50)
    lv = B.Leaves(np.asarray([0, 400, 1000], np.int32), np.arange(N, dtype=np.int32),
                  np.asarray([0, 0], np.int32))
    with pytest.raises(G.GsknnError):
        job.run_pass(lv)
    bad = B.Leaves(np.asarray([0, 3], np.int32), np.asarray([1, 2, N], np.int32),
                   np.asarray([0], np.int32))
    with pytest.raises(G.GsknnError):
        job.run_pass(bad)
    job.close()
