"""The reference's own Python wrapper (python/gsknn.py, unchanged) bound to this library.

The wrapper loads $GSKNN_DIR/lib/libgsknn.so on every call (python/gsknn.py:32-33) and calls
sgsknn_var1 / dgsknn_var1 / sgsknn_ref / dgsknn_ref through ctypes. This test points GSKNN_DIR
at a temporary directory whose lib/libgsknn.so is a link to rnn_b200/libgsknn.so, imports the
wrapper from the reference sources (skipped where they are absent), and checks that each of its
four functions reaches this library: without a GPU every call returns with the library's
status set to a CUDA error and the caller's D/I untouched, never a crash or an exit; with a GPU
the results are checked against the FP64 oracle.
"""
import importlib.util
import os

import numpy as np
import pytest

from rnn_b200 import gsknn as G
from rnn_b200 import workloads as W

REF_WRAPPER = os.path.join(os.environ.get("GSKNN_REFERENCE_DIR", "/root/reference"), "python",
                           "gsknn.py")


@pytest.fixture(scope="module")
def refmod(tmp_path_factory):
    if not os.path.exists(REF_WRAPPER):
        pytest.skip("reference python/gsknn.py not present on this machine")
    d = tmp_path_factory.mktemp("gsknn_dir")
    os.makedirs(d / "lib")
    os.symlink(G.lib()._name, d / "lib" / "libgsknn.so")
    old = os.environ.get("GSKNN_DIR")
    os.environ["GSKNN_DIR"] = str(d)
    spec = importlib.util.spec_from_file_location("reference_gsknn_wrapper", REF_WRAPPER)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    yield mod
    if old is None:
        del os.environ["GSKNN_DIR"]
    else:
        os.environ["GSKNN_DIR"] = old


def _cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.parametrize("fn,dtype", [("sgsknn", np.float32), ("dgsknn", np.float64),
                                      ("sgsknn_ref", np.float32), ("dgsknn_ref", np.float64)])
def test_reference_wrapper_reaches_library(refmod, oracle, fn, dtype):
    # the wrapper asserts D.size == n * d, so d == k here (python/gsknn.py:21-22)
    N, d, k, m, n = 600, 16, 16, 400, 90
    X = W.uniform_table(901, N, d, dtype)
    X2 = W.sq_norms(X)
    r = W.permutation(902, N)[:m].astype(np.int32)
    q = W.permutation(903, N)[:n].astype(np.int32)
    big = 1.79e308 if dtype == np.float64 else 1.79e30
    D = np.full((n, k), big, dtype=dtype)
    I = np.full((n, k), -1, dtype=np.int32)
    getattr(refmod, fn)(d, k, X, X2, q, X, X2, r, D, I)
    code, msg = G.last_error()
    if not _cuda():
        assert code == 3, (code, msg)  # GSKNN_ERR_CUDA: the call reached this library
        assert np.all(I == -1) and np.all(D == big)
        return
    assert code == 0, msg
    from test_gpu_parity import check_against_oracle
    check_against_oracle(oracle, X, X2, r, q, k, D, I, np.full((n, k), big, dtype=dtype),
                         np.full((n, k), -1, dtype=np.int32))
