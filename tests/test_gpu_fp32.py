"""GPU parity of the plain FP32 CUDA-core pipeline (``GSKNN_MODE_FP32``) against the oracle.

In AUTO mode every float call whose shape fits a tensor-core plan takes the precision form, so
the float cases of test_gpu_parity.py exercise the tensor-core path. These tests force FP32 and
check the fused CUDA-core kernel (``pack_panels`` -> ``fused_knn_simt<float>`` with its packed
pair FMAs -> ``finalize_heap``) through ``sgsknn_var1`` / ``sgsknn`` / ``gsknn_s_device``:

  * the reference's golden float cases, every shape of the shape sweep, small-integer data
    (float arithmetic exact: identical (distance, index) rows, lower-index tie rule) and the
    headline workload at full size with sampled rows;
  * each returned distance lies within the FP32 rounding bound of its id's FP64 distance and
    index sets equal the FP64 oracle's except for ids within that bound of the k-th distance
    (``check_against_oracle``);
  * the library's launch tracer shows the CUDA-core kernel ran and the tensor-core one did not.
"""
import json
import ctypes

import numpy as np
import pytest

from knn_check import is_maxheap
from rnn_b200 import gsknn as G
from rnn_b200 import workloads as W
from test_gpu_parity import GOLDEN_CASES, SHAPES, check_against_oracle, run_var1

pytestmark = pytest.mark.gpu


@pytest.fixture
def fp32_mode():
    G.set_mode(G.MODE_FP32)
    L = G.lib()
    L.gsknn_trace_enable(1)
    buf = ctypes.create_string_buffer(1 << 16)
    L.gsknn_trace_read(buf, len(buf))  # drop earlier records
    yield
    L.gsknn_trace_enable(0)
    G.set_mode(G.MODE_AUTO)


def kernels_run():
    """Kernel brackets recorded by the tracer since the last read."""
    import torch
    torch.cuda.synchronize()
    L = G.lib()
    buf = ctypes.create_string_buffer(1 << 16)
    L.gsknn_trace_read(buf, len(buf))
    return set(json.loads(buf.value.decode() or "{}").keys())


def assert_cuda_core_path(k):
    names = kernels_run()
    assert "tc_knn" not in names, names
    if k <= 256:  # lists beyond 256 go to the explicit-distance path
        assert "fused_knn_simt" in names and "finalize_heap" in names, names


@pytest.mark.parametrize("case", [c for c in GOLDEN_CASES if "_s_" in c])
def test_fp32_golden_cases(oracle, golden, fp32_mode, case):
    g = golden(case)
    X, X2, alpha, beta, k = g["X"], g["X2"], g["alpha"], g["beta"], int(g["k"])
    D, I = run_var1(X, X2, alpha, beta, k, g["Din"], g["Iin"])
    assert_cuda_core_path(k)
    check_against_oracle(oracle, X, X2, alpha, beta, k, D, I, g["Din"], g["Iin"],
                         exact_float="ties" in case)


@pytest.mark.parametrize("shape", SHAPES)
def test_fp32_shapes(oracle, fp32_mode, shape):
    m, n, d, k = shape
    N = m + n + 17
    X = W.uniform_table(1000 + m + d, N, d, np.float32)
    X2 = W.sq_norms(X)
    alpha = W.permutation(7 + m, N)[:m].astype(np.int32)
    beta = W.permutation(9 + n, N)[:n].astype(np.int32)
    D, I = run_var1(X, X2, alpha, beta, k)
    assert_cuda_core_path(k)
    Din = np.full((n, k), 1.79e30, dtype=np.float32)
    Iin = np.full((n, k), -1, dtype=np.int32)
    check_against_oracle(oracle, X, X2, alpha, beta, k, D, I, Din, Iin)


@pytest.mark.parametrize("d", [5, 64, 130])
def test_fp32_integer_grid_ties_exact(oracle, fp32_mode, d):
    """Small-integer coordinates make every FP32 product and sum exact, so the CUDA-core
    kernel's rows must equal the oracle's bit for bit, ties to the lower index included."""
    N = 3000
    X = np.floor(W.uniform(77 + d, (N, d)) * 4.0).astype(np.float32)
    X2 = W.sq_norms(X)
    alpha = W.permutation(78, N)[:2500].astype(np.int32)
    beta = W.permutation(79, N)[:700].astype(np.int32)
    for k in (1, 7, 32, 64, 150, 256):
        D, I = run_var1(X, X2, alpha, beta, k)
        assert_cuda_core_path(k)
        Din = np.full((beta.size, k), 1.79e30, dtype=np.float32)
        Iin = np.full((beta.size, k), -1, dtype=np.int32)
        check_against_oracle(oracle, X, X2, alpha, beta, k, D, I, Din, Iin, exact_float=True)


def test_fp32_heap_api_merge(oracle, fp32_mode):
    """sgsknn through heap_t (heapCreate_s), two calls merging into the same heap."""
    N, d, k = 5000, 48, 24
    X = W.gaussian_mixture_table(81, N, d, dtype=np.float32)
    X2 = W.sq_norms(X)
    beta = W.permutation(82, N)[:600].astype(np.int32)
    a1 = W.permutation(83, N)[:2000].astype(np.int32)
    a2 = W.permutation(84, N)[:2000].astype(np.int32)
    h = G.Heap(beta.size, k, 1.79e30, double=False)
    G.gsknn_heap(k, X, X2, a1, X, X2, beta, h)
    D1, I1 = h.D.copy(), h.I.copy()
    G.gsknn_heap(k, X, X2, a2, X, X2, beta, h)
    D2, I2 = h.D.copy(), h.I.copy()
    h.free()
    assert_cuda_core_path(k)
    D0 = np.full((beta.size, k), 1.79e30, dtype=np.float32)
    I0 = np.full((beta.size, k), -1, dtype=np.int32)
    check_against_oracle(oracle, X, X2, a1, beta, k, D1, I1, D0, I0)
    check_against_oracle(oracle, X, X2, a2, beta, k, D2, I2, D1, I1)


def test_fp32_config2_sampled_rows_device_api(oracle, fp32_mode):
    """The headline workload at full size in plain FP32 through gsknn_s_device (N=1,048,576,
    d=64, 65,536 queries x 262,144 references, k=32); 512 sampled rows against the FP64
    oracle within the FP32 bound."""
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
    assert_cuda_core_path(p.k)
    Dh, Ih = D.cpu().numpy(), I.cpu().numpy()
    assert is_maxheap(Dh)
    rows = W.permutation(6, p.n)[:512]
    sub_beta = np.ascontiguousarray(p.beta[rows])
    check_against_oracle(oracle, p.X, p.X2, p.alpha, sub_beta, p.k, Dh[rows], Ih[rows],
                         np.full((512, p.k), np.inf, dtype=np.float32),
                         np.full((512, p.k), -1, dtype=np.int32))
