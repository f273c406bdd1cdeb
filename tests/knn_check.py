"""Comparison helpers for kNN parity: index sets modulo exact or near ties, distance error,
heap validity. Used by the CPU and GPU tests alike."""
from __future__ import annotations

import numpy as np


def exact_dists(X, beta_row_point, ids, X2=None):
    """FP64 squared distances from one query point to table rows `ids` (clamped at 0)."""
    q = X[beta_row_point].astype(np.float64)
    P = X[ids].astype(np.float64)
    if X2 is None:
        qq = q @ q
        pp = np.einsum("ij,ij->i", P, P)
    else:
        qq = float(X2[beta_row_point])
        pp = X2[ids].astype(np.float64)
    return np.maximum(0.0, -2.0 * (P @ q) + pp + qq)


def compare_sets(I_got, I_exp, D_exp, kth_band, dist_of=None):
    """Return (n_rows_equal, bad_rows).

    Rows whose index multisets differ are acceptable only when every differing id lies
    within `kth_band[row]` of the row's expected k-th distance (ties or near-ties at the
    boundary). `dist_of(row, ids)` gives the FP64 distance of ids not in the expected list.
    """
    n, k = I_exp.shape
    bad = []
    equal = 0
    for j in range(n):
        a = np.sort(I_got[j])
        b = np.sort(I_exp[j])
        if np.array_equal(a, b):
            equal += 1
            continue
        kth = D_exp[j].max()
        got_only = np.setdiff1d(a, b)
        exp_only = np.setdiff1d(b, a)
        ok = True
        if exp_only.size:
            de = D_exp[j][np.isin(I_exp[j], exp_only)]
            if np.any(np.abs(de - kth) > kth_band[j]):
                ok = False
        if ok and got_only.size:
            if dist_of is None:
                ok = False
            else:
                dg = dist_of(j, got_only[got_only >= 0])
                if np.any(np.abs(dg - kth) > kth_band[j]):
                    ok = False
                if np.any(got_only < 0) and np.isfinite(kth):
                    ok = False
        if not ok:
            bad.append(j)
    return equal, bad


def is_maxheap(D):
    """Rows of D (n, k) are valid binary max-heaps."""
    n, k = D.shape
    if k < 2:
        return True
    s = np.arange(1, k)
    return bool(np.all(D[:, (s - 1) // 2] >= D[:, s]))


def sorted_rows(D, I):
    """Sort each row by (distance, unsigned index)."""
    Iu = I.astype(np.int64) & 0xFFFFFFFF
    order = np.lexsort((Iu, D), axis=-1)
    return np.take_along_axis(D, order, -1), np.take_along_axis(I, order, -1)
