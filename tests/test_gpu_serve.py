"""GPU tests of the serving form: requests against a resident reference set, continuous
batching on several streams, admission by heap budget, heaps kept on the device.

Every request's result must be the exact FP64 top-k of its queries (ties to the lower id,
the oracle's tie-resolved selection), and identical bit for bit whether the request ran alone
or in a mix with others that arrived while it was queued or running.
"""
import threading
import time

import numpy as np
import pytest

from knn_check import is_maxheap
from rnn_b200 import gsknn as G
from rnn_b200 import serve as S
from rnn_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _refs(seed, n, d):
    import torch
    R = W.uniform_table(seed, n, d).astype(np.float32)
    R2 = W.sq_norms(R)
    return R, R2, torch.from_numpy(R).cuda(), torch.from_numpy(R2).cuda()


def _requests(seed, count, d, ms, ks):
    out = []
    for i in range(count):
        m = ms[i % len(ms)]
        k = ks[(i * 7) % len(ks)]
        out.append((W.uniform_table(seed + 17 * i, m, d).astype(np.float32), k))
    return out


def _check_exact(oracle, R, R2, Q, k, D, I):
    Q2 = W.sq_norms(Q)
    alpha = np.arange(R.shape[0], dtype=np.int32)
    beta = np.arange(Q.shape[0], dtype=np.int32)
    # queries and references in one table for the oracle
    X = np.concatenate([R, Q]).astype(np.float32)
    X2 = np.concatenate([R2, Q2]).astype(np.float32)
    De, Ie = oracle.knn_exact(k, X, X2, alpha, X, X2, beta + R.shape[0], clamp=True)
    assert is_maxheap(D)
    # identical index sets (the FP64 top-k, ties to the lower id); the order inside a row can
    # differ where two FP64 distances round to the same float
    assert np.array_equal(np.sort(I, axis=1), np.sort(Ie, axis=1))
    Ds = np.sort(D.astype(np.float64), axis=1)
    fin = np.isfinite(De)
    assert np.all(np.abs(Ds[fin] - De[fin]) <= 1e-6 * np.abs(De[fin]) + 1e-9)


@pytest.mark.parametrize("mode", [0, 2])
def test_serve_requests_are_exact(oracle, mode):
    R, R2, Rd, R2d = _refs(1000, 30000, 128)
    srv = S.Server(Rd, R2d, mode=mode, max_batch_queries=2048, max_k=64, heap_budget=64 << 20,
                   slots=2)
    # 2500 rows: more than a batch holds, served in pieces
    reqs = _requests(1001, 7, 128, [1, 7, 130, 600, 1000, 2048, 2500], [8, 16, 64])
    ids = [srv.submit(Q, k) for Q, k in reqs]
    for rid, (Q, k) in zip(ids, reqs):
        srv.wait(rid)
        D, I = srv.fetch(rid)
        _check_exact(oracle, R, R2, Q, k, D, I)
        srv.release(rid)
    srv.close()


def test_serve_same_alone_and_in_the_mix():
    """Each request alone (waited before the next), then all of them arriving at random
    moments from two client threads while others run: identical heaps bit for bit."""
    R, R2, Rd, R2d = _refs(1010, 40000, 64)
    srv = S.Server(Rd, R2d, mode=0, max_batch_queries=4096, max_k=64, heap_budget=256 << 20,
                   slots=3)
    reqs = _requests(1011, 24, 64, [1, 3, 40, 257, 900, 2000, 4000], [8, 16, 64])
    alone = []
    for Q, k in reqs:
        rid = srv.submit(Q, k)
        srv.wait(rid)
        alone.append(srv.fetch(rid))
        srv.release(rid)
    ids = [None] * len(reqs)
    rng = np.random.default_rng(5)
    gaps = rng.exponential(0.002, size=len(reqs))

    def client(parity):
        for i in range(parity, len(reqs), 2):
            time.sleep(gaps[i])
            ids[i] = srv.submit(*reqs[i])

    th = [threading.Thread(target=client, args=(p,)) for p in (0, 1)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i, rid in enumerate(ids):
        srv.wait(rid)
        D, I = srv.fetch(rid)
        assert np.array_equal(D, alone[i][0]), i
        assert np.array_equal(I, alone[i][1]), i
        srv.release(rid)
    # a burst queued while dispatch is held: packed into shared batches, same results
    srv.pause(True)
    ids = [srv.submit(Q, k) for Q, k in reqs]
    srv.pause(False)
    batches = set()
    for i, rid in enumerate(ids):
        srv.wait(rid)
        D, I = srv.fetch(rid)
        batches.add(srv.stats(rid)["batch"])
        assert np.array_equal(D, alone[i][0]), i
        assert np.array_equal(I, alone[i][1]), i
        srv.release(rid)
    assert len(batches) < len(reqs)
    srv.close()


def test_serve_admission_waits_for_heap_budget():
    """Budget for two heaps: the third request waits until a finished one is released."""
    R, R2, Rd, R2d = _refs(1020, 20000, 32)
    m, k = 512, 16
    per = m * k * 8
    srv = S.Server(Rd, R2d, mode=0, max_batch_queries=1024, max_k=16, heap_budget=2 * per,
                   slots=2)
    Qs = [W.uniform_table(1021 + i, m, 32).astype(np.float32) for i in range(3)]
    a = srv.submit(Qs[0], k)
    b = srv.submit(Qs[1], k)
    srv.wait(a)
    srv.wait(b)
    c = srv.submit(Qs[2], k)
    time.sleep(0.5)
    assert srv.test(c) == 0  # no heap memory left: still queued
    srv.release(a)
    srv.wait(c, timeout=30)
    D, I = srv.fetch(c)
    assert np.all(I >= 0)
    srv.release(b)
    srv.release(c)
    srv.close()


def test_serve_rejects_requests_beyond_its_limits():
    R, R2, Rd, R2d = _refs(1030, 5000, 16)
    srv = S.Server(Rd, R2d, mode=0, max_batch_queries=256, max_k=16, heap_budget=1 << 20,
                   slots=1)
    with pytest.raises(G.GsknnError):
        srv.submit(np.zeros((20000, 16), np.float32), 8)  # heap above the whole budget
    with pytest.raises(G.GsknnError):
        srv.submit(np.zeros((10, 16), np.float32), 32)   # k above max_k
    srv.close()


def test_serve_slices_do_not_change_results():
    """The same requests with whole batches and with 128-row slices (large requests in up to
    32 pieces): identical heaps bit for bit."""
    R, R2, Rd, R2d = _refs(1040, 40000, 64)
    srv = S.Server(Rd, R2d, mode=0, max_batch_queries=4096, max_k=64, heap_budget=256 << 20,
                   slots=2)
    assert srv.slice_rows == 4096  # default for this small reference set: the whole batch
    reqs = _requests(1041, 9, 64, [1, 130, 900, 2000, 4000, 5000], [8, 16, 64])
    out = {}
    for rows in (4096, 128):
        assert srv.set_slice(rows) == rows
        srv.pause(True)
        ids = [srv.submit(Q, k) for Q, k in reqs]
        srv.pause(False)
        res = []
        for rid in ids:
            srv.wait(rid, timeout=60)
            res.append(srv.fetch(rid))
            srv.release(rid)
        out[rows] = res
    for (D0, I0), (D1, I1) in zip(out[4096], out[128]):
        assert np.array_equal(D0, D1) and np.array_equal(I0, I1)
    assert srv.set_slice(0) == 4096 and srv.set_slice(200) == 256
    srv.close()


def test_serve_small_request_shares_the_first_slice_of_a_large_one():
    """A large request queued first and a small one behind it: the first batch holds the small
    request whole and a piece of the large one, so the small one finishes first."""
    R, R2, Rd, R2d = _refs(1050, 60000, 64)
    srv = S.Server(Rd, R2d, mode=0, max_batch_queries=4096, max_k=64, heap_budget=256 << 20,
                   slots=1, slice_rows=512)
    big = W.uniform_table(1051, 4000, 64).astype(np.float32)
    small = W.uniform_table(1052, 3, 64).astype(np.float32)
    srv.pause(True)
    b = srv.submit(big, 16)
    a = srv.submit(small, 16)
    srv.pause(False)
    srv.wait(a, timeout=60)
    srv.wait(b, timeout=60)
    sa, sb = srv.stats(a), srv.stats(b)
    assert sa["batch"] == sb["batch"]          # both start in the first batch
    assert sa["batch_rows"] == 512             # 3 rows + a 509-row piece of the large one
    assert sa["total_ms"] < sb["total_ms"]
    srv.release(a)
    srv.release(b)
    srv.close()
