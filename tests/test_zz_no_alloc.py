"""gsknn_s_device_noalloc: the fused-kNN entry point for callers that cannot allocate GPU memory
while they run (a program that pre-reserves the GPU's memory for its own pool, a latency-bound
serving loop, a plugin host that forbids device allocations). Its scratch lives in a fixed array
inside the library, so the call itself must not allocate.

Checked through the C ABI against the caching entry point gsknn_s_device, on two calls in a row
(the second merges a fresh candidate set into the heaps the first produced, so stale contents
of the shared scratch would show). This file is collected last; it passes alone in a fresh
process and after the other tests."""
import ctypes

import numpy as np
import pytest

from rnn_b200 import gsknn as G
from rnn_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6  # float tolerance on distances; index sets must be identical


def _bind():
    L = G.lib()
    f = L.gsknn_s_device_noalloc
    vp, ci, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
    f.argtypes = [ci, ci, ci, ci, vp, vp, ll, vp, vp, vp, ll, vp, vp, vp, ci, vp, vp]
    f.restype = ci
    return L, f


def _call_existing(L, X, X2, alpha, beta, D, I, st):
    rc = L.gsknn_s_device(alpha.numel(), beta.numel(), X.shape[1], D.shape[1], X.data_ptr(),
                          X2.data_ptr(), X.shape[0], alpha.data_ptr(), X.data_ptr(),
                          X2.data_ptr(), X.shape[0], beta.data_ptr(), D.data_ptr(), I.data_ptr(),
                          D.stride(0), st.cuda_stream)
    assert rc == 0, G.last_error()


def _call_noalloc(f, X, X2, alpha, beta, D, I, status, st):
    return f(alpha.numel(), beta.numel(), X.shape[1], D.shape[1], X.data_ptr(), X2.data_ptr(),
             X.shape[0], alpha.data_ptr(), X.data_ptr(), X2.data_ptr(), X.shape[0],
             beta.data_ptr(), D.data_ptr(), I.data_ptr(), D.stride(0),
             None if status is None else status.data_ptr(), st.cuda_stream)


def _same(Da, Ia, Db, Ib):
    Ia, Ib = Ia.cpu().numpy(), Ib.cpu().numpy()
    Da, Db = Da.cpu().numpy().astype(np.float64), Db.cpu().numpy().astype(np.float64)
    assert np.array_equal(np.sort(Ia, axis=1), np.sort(Ib, axis=1))
    sa, sb = np.sort(Da, axis=1), np.sort(Db, axis=1)
    fin = np.isfinite(sa)
    assert np.array_equal(fin, np.isfinite(sb))
    assert np.all(np.abs(sa[fin] - sb[fin]) <= REL_TOL * np.maximum(np.abs(sb[fin]), 1e-30))
    assert np.all(Da[:, :-1] >= Da[:, 1:])  # rows stay max-heaps (descending)


def test_noalloc_matches_caching_entry_point_two_calls():
    # the no-alloc variant runs the CUDA-core FP32 pipeline: compare with gsknn_s_device in
    # the same arithmetic
    prev = G.get_mode()
    G.set_mode(G.MODE_FP32)
    try:
        _compare_two_calls()
    finally:
        G.set_mode(prev)


def _compare_two_calls():
    import torch
    L, f = _bind()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    st = torch.cuda.current_stream(dev)
    N, d, k = 60000, 48, 24
    X = torch.from_numpy(W.gaussian_mixture_table(31, N, d, dtype=np.float32)).to(dev)
    X2 = (X.double() ** 2).sum(1).float()
    beta = torch.from_numpy(W.permutation(32, N)[:3000].astype(np.int32)).to(dev)
    alphas = [torch.from_numpy(W.permutation(33 + c, N)[:20000].astype(np.int32)).to(dev)
              for c in range(2)]
    n = beta.numel()
    D_ref = torch.full((n, k), float("inf"), device=dev)
    I_ref = torch.full((n, k), -1, dtype=torch.int32, device=dev)
    D_na = D_ref.clone()
    I_na = I_ref.clone()
    status = torch.full((1,), 12345, dtype=torch.int32, device=dev)

    # first call: sets up the scratch address for this device
    _call_existing(L, X, X2, alphas[0], beta, D_ref, I_ref, st)
    rc = _call_noalloc(f, X, X2, alphas[0], beta, D_na, I_na, status, st)
    assert rc == 0, G.last_error()
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    _same(D_na, I_na, D_ref, I_ref)

    # second call in a row: no device memory may be taken by the call
    _call_existing(L, X, X2, alphas[1], beta, D_ref, I_ref, st)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    rc = _call_noalloc(f, X, X2, alphas[1], beta, D_na, I_na, status, st)
    assert rc == 0, G.last_error()
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info(dev)[0]
    assert free_after >= free_before
    assert int(status.item()) == 0
    _same(D_na, I_na, D_ref, I_ref)


def test_noalloc_rejects_problems_beyond_its_scratch():
    import torch
    L, f = _bind()
    dev = torch.device("cuda:0")
    st = torch.cuda.current_stream(dev)
    # 2M candidates x d=64 needs ~512 MiB of panels: must be refused before any launch
    X = torch.zeros((16, 64), device=dev)
    X2 = torch.zeros(16, device=dev)
    alpha = torch.zeros(2_000_000, dtype=torch.int32, device=dev)
    beta = torch.zeros(8, dtype=torch.int32, device=dev)
    D = torch.full((8, 4), float("inf"), device=dev)
    I = torch.full((8, 4), -1, dtype=torch.int32, device=dev)
    rc = _call_noalloc(f, X, X2, alpha, beta, D, I, None, st)
    assert rc == 5  # GSKNN_ERR_UNSUPPORTED
    assert "fixed scratch" in G.last_error()[1]
    torch.cuda.synchronize()
    assert torch.all(I == -1)


def test_noalloc_reports_out_of_range_index_and_rejects_large_k():
    """An alpha/beta entry outside its table reaches the caller's status word (and is never
    read); k beyond the fused kernel's list size is refused before any launch."""
    import torch
    L, f = _bind()
    dev = torch.device("cuda:0")
    st = torch.cuda.current_stream(dev)
    N, d = 500, 16
    X = torch.rand((N, d), device=dev)
    X2 = (X.double() ** 2).sum(1).float()
    alpha = torch.arange(300, dtype=torch.int32, device=dev)
    beta = torch.arange(300, 340, dtype=torch.int32, device=dev)
    beta[5] = N  # one past the end of the table
    D = torch.full((40, 8), float("inf"), device=dev)
    I = torch.full((40, 8), -1, dtype=torch.int32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    rc = _call_noalloc(f, X, X2, alpha, beta, D, I, status, st)
    assert rc == 0, G.last_error()
    torch.cuda.synchronize()
    assert int(status.item()) == 4  # GSKNN_ERR_INDEX
    beta[5] = 5
    D300 = torch.full((40, 300), float("inf"), device=dev)
    I300 = torch.full((40, 300), -1, dtype=torch.int32, device=dev)
    rc = _call_noalloc(f, X, X2, alpha, beta, D300, I300, status, st)
    assert rc == 5  # GSKNN_ERR_UNSUPPORTED
    torch.cuda.synchronize()
    assert torch.all(I300 == -1) and torch.all(torch.isinf(D300))
