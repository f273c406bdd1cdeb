"""Generate the golden fixtures under tests/golden/ from the reference GSKNN library.

The reference ships no golden vectors or known-answer tests (its test drivers compare against
its own in-repo oracle on random data and print mismatches). These fixtures are outputs of the
reference library itself, compiled from its sources by oracle/Makefile (`make -C oracle ref`),
on seeded inputs from rnn_b200.workloads. They pin the oracle restatement (oracle/) and give
the CUDA parity tests fixed expectations. Regenerate with:

    make -C oracle ref && python tests/golden/make_golden.py            # every case
    make -C oracle ref && python tests/golden/make_golden.py --only l1  # the 1-norm cases

Each case is one .npz with the inputs (or, for the full-size config-1 case, a checksum of the
regenerated inputs) and the reference outputs.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import ReferenceLib  # noqa: E402
from rnn_b200 import workloads as W  # noqa: E402


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def save(name, **kw):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **kw)
    print(f"{name}: {os.path.getsize(path)} bytes")


def ref_oracle_case(ref, name, seed, N, d, m, n, k, dtype, table="uniform", stl=False,
                    prefill=False):
    """dgsknn_ref / sgsknn_ref on a seeded table (frame/gsknn_ref.c)."""
    if table == "uniform":
        X = W.uniform_table(seed, N, d, dtype)
    elif table == "grid":  # integer coordinates: many exact ties and duplicate points
        X = np.floor(W.uniform(seed, (N, d)) * 3.0).astype(dtype)
    else:
        X = W.gaussian_mixture_table(seed, N, d, dtype=dtype)
    X2 = W.sq_norms(X)
    alpha = W.permutation(seed + 1, N)[:m].astype(np.int32)
    beta = W.permutation(seed + 2, N)[:n].astype(np.int32)
    big = 1.79e308 if dtype == np.float64 else 1.79e30
    Din = np.full((n, k), big, dtype=dtype)
    Iin = np.full((n, k), -1, dtype=np.int32)
    if prefill:
        # A valid incoming heap from an earlier call over other candidates.
        pre = W.permutation(seed + 3, N)[:max(k, 8)].astype(np.int32)
        ref.gsknn_ref(k, X, X2, pre, X, X2, beta, Din, Iin)
    Dout, Iout = Din.copy(), Iin.copy()
    ref.gsknn_ref(k, X, X2, alpha, X, X2, beta, Dout, Iout, stl=stl)
    save(name, kind="gsknn_ref" + ("_stl" if stl else ""), k=k, X=X, X2=X2, alpha=alpha,
         beta=beta, Din=Din, Iin=Iin, Dout=Dout, Iout=Iout)


def optimized_case(ref, name, seed, N, d, m, n, k, dtype, table="uniform", calls=1):
    """The optimized dgsknn / sgsknn through heap_t (frame/gsknn.c:1106-1184), `calls`
    successive calls with fresh candidate sets merging into the same heap."""
    if table == "uniform":
        X = W.uniform_table(seed, N, d, dtype)
    else:
        X = W.gaussian_mixture_table(seed, N, d, dtype=dtype)
    X2 = W.sq_norms(X)
    beta = W.permutation(seed + 2, N)[:n].astype(np.int32)
    dbl = dtype == np.float64
    big = 1.79e308 if dbl else 1.79e30
    h = ref.heap_create(n, k, big, double=dbl)
    D, I = ref.heap_arrays(h, double=dbl)
    Din, Iin = D.copy(), I.copy()
    alphas, outs_D, outs_I = [], [], []
    for c in range(calls):
        alpha = W.permutation(seed + 10 + c, N)[:m].astype(np.int32)
        ref.gsknn(k, X, X2, alpha, X, X2, beta, h)
        alphas.append(alpha)
        outs_D.append(D.copy())
        outs_I.append(I.copy())
    ref.heap_free(h, double=dbl)
    save(name, kind="gsknn", k=k, X=X, X2=X2, beta=beta, alphas=np.stack(alphas),
         Din=Din, Iin=Iin, Douts=np.stack(outs_D), Iouts=np.stack(outs_I))


def config1_case(ref, seed=1):
    """Config 1 at full size: dgsknn f64, N=8192, d=32, m=n=4096, k=16, two calls; outputs of
    both the optimized dgsknn and dgsknn_ref. Inputs are regenerated from the seed."""
    p, alpha2 = W.config1(seed)
    X, X2 = p.X, p.X2
    h = ref.heap_create(p.n, p.k, 1.79e308)
    D, I = ref.heap_arrays(h)
    ref.gsknn(p.k, X, X2, p.alpha, X, X2, p.beta, h)
    D1, I1 = D.copy(), I.copy()
    ref.gsknn(p.k, X, X2, alpha2, X, X2, p.beta, h)
    D2, I2 = D.copy(), I.copy()
    ref.heap_free(h)
    Dr = np.full((p.n, p.k), 1.79e308)
    Ir = np.full((p.n, p.k), -1, dtype=np.int32)
    ref.gsknn_ref(p.k, X, X2, p.alpha, X, X2, p.beta, Dr, Ir)
    Dr1, Ir1 = Dr.copy(), Ir.copy()
    ref.gsknn_ref(p.k, X, X2, alpha2, X, X2, p.beta, Dr, Ir)
    save("config1_dgsknn", kind="config1", seed=seed, k=p.k,
         input_sha256=digest(X, X2, p.alpha, p.beta, alpha2),
         D1=D1, I1=I1, D2=D2, I2=I2, Dref1=Dr1, Iref1=Ir1, Dref2=Dr, Iref2=Ir)


def var3_case(ref, seed=21):
    """dgsknn with k=600 > KNN_VAR_THRES: heapCreate_d's 4-ary header layout
    (frame/gsknn_heap.c:257-307) and dgsknn_var3 (frame/gsknn.c:597-659); three calls so the
    heap goes through partial fill, fill completion and replacement."""
    N, d, n, k = 2048, 16, 32, 600
    X = W.uniform_table(seed, N, d)
    X2 = W.sq_norms(X)
    beta = W.permutation(seed + 1, N)[:n].astype(np.int32)
    h = ref.heap_create(n, k, 1.79e308)
    D, I = ref.heap_arrays(h)
    Din, Iin = D.copy(), I.copy()
    alphas, Ds, Is = [], [], []
    for c, m in enumerate((300, 500, 1024)):
        alpha = W.permutation(seed + 10 + c, N)[:m].astype(np.int32)
        ref.gsknn(k, X, X2, alpha, X, X2, beta, h)
        alphas.append(np.pad(alpha, (0, 1024 - m), constant_values=-1))
        Ds.append(D.copy())
        Is.append(I.copy())
    ref.heap_free(h)
    save("var3_k600", kind="var3", k=k, X=X, X2=X2, beta=beta, alphas=np.stack(alphas),
         ms=np.array([300, 500, 1024]), Din=Din, Iin=Iin, Douts=np.stack(Ds), Iouts=np.stack(Is))


def sq2nrm_case(ref, seed=31):
    N, d, m, n = 300, 300, 37, 23
    X = W.uniform_table(seed, N, d)
    X2 = W.sq_norms(X)
    amap = W.permutation(seed + 1, N)[:m].astype(np.int32)
    bmap = W.permutation(seed + 2, N)[:n].astype(np.int32)
    C = ref.dgssq2nrm(X, X2, amap, X, X2, bmap, ldc=40)
    save("dgssq2nrm_d300", kind="dgssq2nrm", X=X, X2=X2, amap=amap, bmap=bmap, ldc=40,
         C=C[:, :m])


def heapselect_case(ref, seed=41):
    """heapSelect_d / heapSelect_s on a prefilled heap (frame/gsknn_heap.c:104-162)."""
    out = {}
    for tag, dt in (("d", np.float64), ("s", np.float32)):
        k, m = 13, 200
        keys = W.uniform(seed, (m,)).astype(dt)
        keys[50:60] = keys[10]  # ties
        alpha = (np.arange(m) * 7 + 3).astype(np.int32)
        D = np.sort(W.uniform(seed + 1, (k,)).astype(dt))[::-1].copy()  # descending: a heap
        I = np.arange(100, 100 + k, dtype=np.int32)
        out[f"keys_{tag}"], out[f"alpha_{tag}"] = keys, alpha
        out[f"Din_{tag}"], out[f"Iin_{tag}"] = D.copy(), I.copy()
        ref.heap_select(keys, alpha, D, I)
        out[f"Dout_{tag}"], out[f"Iout_{tag}"] = D, I
    save("heapselect", kind="heapselect", **out)


def l1_case(name, seed, m, n, d, k, table="uniform"):
    """The reference's 1-norm micro-kernel (kernels/x86_64/sandybridge/rnn_r_1norm_int_d8x4_row.c)
    over every 8 x 4 block, driven by oracle/ref_l1_harness.c, into heaps initialised as
    heapCreate_d does (DBL_MAX, -1): m queries XQ against n candidates XC."""
    import ctypes
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_l1.so"))
    if table == "grid":  # small integer coordinates: many exact ties
        XQ = W.randint(seed, m * d, 5).reshape(m, d).astype(np.float64)
        XC = W.randint(seed + 1, n * d, 5).reshape(n, d).astype(np.float64)
    else:
        XQ = W.uniform_table(seed, m, d)
        XC = W.uniform_table(seed + 1, n, d)
    D = np.full((m, k), np.finfo(np.float64).max)
    I = np.full((m, k), -1, dtype=np.int32)
    Din, Iin = D.copy(), I.copy()
    vp, ci = ctypes.c_void_p, ctypes.c_int
    rc = lib.ref_l1_knn(ci(m), ci(n), ci(d), ci(k), vp(XQ.ctypes.data), vp(XC.ctypes.data),
                        vp(D.ctypes.data), vp(I.ctypes.data))
    assert rc == 0
    save(name, kind="l1", k=k, XQ=XQ, XC=XC, Din=Din, Iin=Iin, Dout=D, Iout=I)


def l1_cases():
    l1_case("l1_d_basic", 301, 120, 500, 7, 5)
    l1_case("l1_d_ties", 302, 90, 300, 3, 8, table="grid")
    l1_case("l1_d_odd", 303, 31, 257, 33, 7)
    l1_case("l1_d_few", 304, 20, 5, 6, 16)
    l1_case("l1_d_dim1", 305, 17, 101, 1, 4)


def main():
    if not ReferenceLib.available():
        sys.exit("reference library missing: run `make -C oracle ref` first")
    if "--only" in sys.argv and sys.argv[sys.argv.index("--only") + 1] == "l1":
        l1_cases()
        return
    ref = ReferenceLib()
    ref_oracle_case(ref, "ref_d_basic", 101, 500, 7, 120, 60, 5, np.float64)
    ref_oracle_case(ref, "ref_s_basic", 102, 500, 7, 120, 60, 5, np.float32)
    ref_oracle_case(ref, "ref_d_prefill", 103, 700, 9, 200, 50, 16, np.float64, prefill=True)
    ref_oracle_case(ref, "ref_s_gmm_d64", 104, 1536, 64, 1024, 128, 32, np.float32, table="gmm")
    ref_oracle_case(ref, "ref_d_ties", 105, 400, 3, 300, 40, 8, np.float64, table="grid")
    ref_oracle_case(ref, "ref_s_ties", 106, 400, 3, 300, 40, 8, np.float32, table="grid")
    ref_oracle_case(ref, "ref_d_few", 107, 64, 5, 5, 20, 16, np.float64)
    ref_oracle_case(ref, "ref_d_odd", 108, 300, 33, 31, 9, 7, np.float64)
    ref_oracle_case(ref, "ref_s_odd", 109, 600, 1, 257, 255, 64, np.float32)
    ref_oracle_case(ref, "ref_d_one", 110, 3, 1, 1, 1, 1, np.float64)
    ref_oracle_case(ref, "ref_d_stl", 111, 500, 7, 120, 60, 5, np.float64, stl=True)
    optimized_case(ref, "opt_d_merge", 201, 2048, 32, 512, 256, 16, np.float64, calls=2)
    optimized_case(ref, "opt_s_gmm", 202, 1536, 64, 1024, 128, 32, np.float32, table="gmm")
    optimized_case(ref, "opt_d_d300", 203, 320, 300, 256, 64, 8, np.float64)
    optimized_case(ref, "opt_s_d300", 204, 320, 300, 256, 64, 8, np.float32)
    config1_case(ref)
    var3_case(ref)
    sq2nrm_case(ref)
    heapselect_case(ref)
    l1_cases()


if __name__ == "__main__":
    main()
