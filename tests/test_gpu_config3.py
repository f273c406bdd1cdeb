"""The precision form on its own workload, at full size: 32,768 queries x 262,144 references,
d = 256, k = 64, points on an 8-dim latent manifold (U[0,1)^8 through a seeded orthonormal
basis into R^256) plus N(0, 1e-3^2) noise, so that near-boundary distances are dense.

For each tensor-core arithmetic (TF32, BF16, split BF16):
  * the full call (all 32,768 queries, through gsknn_s_device) returns, on 512 sampled rows,
    exactly the FP64 oracle's index sets (the semantics of dgsknn_ref, frame/gsknn_ref.c:112-162,
    on the float inputs upcast to double with the caller's norms; ties to the lower index), with
    distances equal to the FP64 values rounded to float;
  * the approximate distance block of 512 queries against all 262,144 references lies within
    the stated bound E of the FP64 value for every pair; max(err / E) is printed.
"""
import ctypes

import numpy as np
import pytest

from knn_check import is_maxheap
from rnn_b200 import gsknn as G
from rnn_b200 import workloads as W
from test_gpu_tc import MODES, _bind, assert_close, assert_same_sets

pytestmark = pytest.mark.gpu

N_SAMPLE = 512


@pytest.fixture(scope="module")
def cfg3():
    import torch
    p = W.config3()
    dev = torch.device("cuda:0")
    t = dict(X=torch.from_numpy(p.X).to(dev), X2=torch.from_numpy(p.X2).to(dev),
             alpha=torch.from_numpy(p.alpha).to(dev), beta=torch.from_numpy(p.beta).to(dev))
    rows = np.sort(W.permutation(33, p.n)[:N_SAMPLE])
    return p, t, rows


@pytest.fixture(scope="module")
def cfg3_exact(cfg3, oracle):
    p, _, rows = cfg3
    sub = np.ascontiguousarray(p.beta[rows])
    De, Ie = oracle.knn_exact(p.k, p.X, p.X2, p.alpha, p.X, p.X2, sub,
                              np.full((N_SAMPLE, p.k), np.inf, dtype=np.float32),
                              np.full((N_SAMPLE, p.k), -1, dtype=np.int32), clamp=True)
    return De, Ie


@pytest.mark.parametrize("mode", ["tf32", "bf16", "bf16x3"])
def test_config3_full_call_exact_sets(cfg3, cfg3_exact, mode):
    import torch
    p, t, rows = cfg3
    De, Ie = cfg3_exact
    dev = t["X"].device
    D = torch.full((p.n, p.k), float("inf"), device=dev)
    I = torch.full((p.n, p.k), -1, dtype=torch.int32, device=dev)
    G.set_mode(MODES[mode])
    try:
        G.knn_device(t["X"], t["X2"], t["alpha"], t["X"], t["X2"], t["beta"], D, I)
    finally:
        G.set_mode(G.MODE_AUTO)
    Dh, Ih = D.cpu().numpy(), I.cpu().numpy()
    assert is_maxheap(Dh)
    sub = np.ascontiguousarray(p.beta[rows])
    assert_same_sets(p.X, p.X2, sub, Ih[rows], Ie, De)
    assert_close(np.sort(Dh[rows].astype(np.float64), axis=1), De)
    rel = np.abs(np.sort(Dh[rows].astype(np.float64), axis=1) - De) / np.maximum(De, 1e-30)
    print(f"config 3 {mode}: 512 rows identical to FP64; max rel dist err {rel.max():.3e}")


@pytest.mark.parametrize("mode", ["tf32", "bf16", "bf16x3"])
def test_config3_distance_block_within_bound(cfg3, mode):
    """Every approximate distance of 512 queries against all references within E; the
    observed max(err / E) is printed (1 would mean the bound is tight)."""
    import torch
    p, t, rows = cfg3
    dev = t["X"].device
    f = _bind()
    sub = torch.from_numpy(np.ascontiguousarray(p.beta[rows])).to(dev)
    m, n, k = p.m, N_SAMPLE, p.k
    Dd = torch.full((n, k), float("inf"), device=dev)
    Id = torch.full((n, k), -1, dtype=torch.int32, device=dev)
    C = torch.full((n, m), float("nan"), device=dev)
    margin = torch.zeros(n, device=dev)
    st = torch.cuda.current_stream(dev)
    N = p.X.shape[0]
    rc = f(MODES[mode], m, n, p.d, k, t["X"].data_ptr(), t["X2"].data_ptr(), N,
           t["alpha"].data_ptr(), t["X"].data_ptr(), t["X2"].data_ptr(), N, sub.data_ptr(),
           Dd.data_ptr(), Id.data_ptr(), k, C.data_ptr(), m, margin.data_ptr(), st.cuda_stream)
    assert rc == 0, G.last_error()
    assert G.lib().gsknn_stream_status(ctypes.c_void_p(st.cuda_stream)) == 0, G.last_error()
    # FP64 block of the float inputs with the caller's norms (unclamped, as d' is)
    Xq = t["X"][sub.long()].double()
    Xc = t["X"][t["alpha"].long()].double()
    exu = (-2.0 * Xq @ Xc.T) + t["X2"][t["alpha"].long()].double()[None, :] \
        + t["X2"][sub.long()].double()[:, None]
    assert bool(torch.isfinite(C).all())
    E = (margin.double() / 2.0)[:, None]
    ratio = ((C.double() - exu).abs() / E).max().item()
    print(f"config 3 {mode}: max |d' - d| / E = {ratio:.4f} over {n} x {m} pairs")
    assert ratio <= 1.0
