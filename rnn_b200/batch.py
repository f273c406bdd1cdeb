"""Batching form: all-nearest-neighbour search over randomized-tree leaves.

The reference's tree drivers call `dgsknn` once per leaf with alpha = beta = the leaf's point
list, merging into per-point heaps. Here every leaf of a pass (the leaves of several trees over
the same points) runs in one persistent launch, replayed from a CUDA graph for every pass, and
the pass's lists are merged into the device heaps with duplicates removed (C ABI:
`gsknn_batch_*`, `gsknn_rkdt_leaves` in include/gsknn.h).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from rnn_b200 import gsknn as G

SHAPES = {0: "128-row tiles, 8x8 per thread", 1: "64-row tiles, 8x4 per thread",
          2: "64-row tiles, 4x4 per thread"}


@dataclass
class Leaves:
    """Leaves of one or more trees over the same points (CSR): leaf l holds
    pts[ptr[l]:ptr[l+1]] and belongs to tree `tree[l]`."""
    ptr: np.ndarray   # int32 [nleaves + 1]
    pts: np.ndarray   # int32
    tree: np.ndarray  # int32 [nleaves]

    @property
    def nleaves(self) -> int:
        return int(self.tree.size)

    def tree_range(self, a: int, b: int) -> "Leaves":
        """Trees [a, b) of a build whose trees are stored one after another (as
        rkdt_leaves returns them), renumbered 0..b-a-1."""
        sel = np.nonzero((self.tree >= a) & (self.tree < b))[0]
        if sel.size == 0:
            return Leaves(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
        l0, l1 = int(sel[0]), int(sel[-1]) + 1
        assert np.array_equal(sel, np.arange(l0, l1)), "trees are not stored contiguously"
        p0, p1 = int(self.ptr[l0]), int(self.ptr[l1])
        return Leaves((self.ptr[l0:l1 + 1] - p0).astype(np.int32), self.pts[p0:p1],
                      (self.tree[l0:l1] - a).astype(np.int32))

    def select_trees(self, trees) -> "Leaves":
        """The leaves of the given trees, renumbered 0..len(trees)-1 in that order."""
        parts_ptr, parts_pts, parts_tree = [0], [], []
        off = 0
        for new_t, t in enumerate(trees):
            sel = np.nonzero(self.tree == t)[0]
            for l in sel:
                seg = self.pts[self.ptr[l]:self.ptr[l + 1]]
                parts_pts.append(seg)
                off += seg.size
                parts_ptr.append(off)
                parts_tree.append(new_t)
        return Leaves(np.asarray(parts_ptr, dtype=np.int32),
                      np.concatenate(parts_pts).astype(np.int32) if parts_pts
                      else np.zeros(0, np.int32),
                      np.asarray(parts_tree, dtype=np.int32))


def rkdt_leaves(X: np.ndarray, ntrees: int, leaf_min: int, leaf_max: int, seed: int,
                threads: int = 0) -> Leaves:
    """Randomized projection trees on the host (`gsknn_rkdt_leaves`): leaf sizes uniform in
    [leaf_min, leaf_max], random Gaussian split directions, trees built in parallel."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    N, d = X.shape
    L = G.lib()
    cap = ntrees * ((N + leaf_min - 1) // leaf_min + 1)
    ptr = np.zeros(cap + 1, dtype=np.int32)
    pts = np.zeros(ntrees * N, dtype=np.int32)
    tree = np.zeros(cap, dtype=np.int32)
    n = ctypes.c_int(0)
    f = L.gsknn_rkdt_leaves
    ci, vp = ctypes.c_int, ctypes.c_void_p
    f.argtypes = [vp, ci, ci, ci, ci, ci, ctypes.c_ulonglong, ci, vp, vp, vp, ci,
                  ctypes.POINTER(ci)]
    rc = f(X.ctypes.data, N, d, ntrees, leaf_min, leaf_max, seed, threads, ptr.ctypes.data,
           pts.ctypes.data, tree.ctypes.data, cap, ctypes.byref(n))
    if rc != 0:
        raise G.GsknnError(rc, G.last_error())
    m = n.value
    return Leaves(ptr[:m + 1].copy(), pts, tree[:m].copy())


class BatchJob:
    """All-nearest-neighbour job on the device (`gsknn_batch_create`).

    X, X2, D, I are CUDA tensors (float32 N x d, float32 N, float32 N x ldD, int32 N x ldD);
    the heap D / I is updated in place by every pass. `shape=-1` lets the autotuner pick the
    tile shape on the first pass of each (d, k, mean leaf size) class."""

    def __init__(self, X, X2, D, I, k: int, trees_per_pass: int, leaf_min: int, shape: int = -1,
                 stream=None):
        import torch
        self._keep = (X, X2, D, I)
        N, d = X.shape
        self.N, self.d, self.k = N, d, k
        self.stream = stream if stream is not None else torch.cuda.current_stream(X.device)
        L = G.lib()
        vp, ci = ctypes.c_void_p, ctypes.c_int
        L.gsknn_batch_create.restype = vp
        L.gsknn_batch_create.argtypes = [ci, ci, ci, vp, vp, vp, vp, ci, ci, ci, ci, vp]
        L.gsknn_batch_pass.argtypes = [vp, vp, vp, vp, ci]
        L.gsknn_batch_sync.argtypes = [vp]
        L.gsknn_batch_destroy.argtypes = [vp]
        L.gsknn_batch_info.argtypes = [vp] + [vp] * 7
        self._L = L
        h = L.gsknn_batch_create(N, d, k, X.data_ptr(), X2.data_ptr(), D.data_ptr(),
                                 I.data_ptr(), D.stride(0), trees_per_pass, leaf_min, shape,
                                 self.stream.cuda_stream)
        if not h:
            raise G.GsknnError(L.gsknn_last_error(), G.last_error())
        self._h = h

    def run_pass(self, leaves: Leaves) -> None:
        """Enqueue one pass over these leaves (asynchronous on the job's stream)."""
        ptr = np.ascontiguousarray(leaves.ptr, dtype=np.int32)
        pts = np.ascontiguousarray(leaves.pts, dtype=np.int32)
        tree = np.ascontiguousarray(leaves.tree, dtype=np.int32)
        rc = self._L.gsknn_batch_pass(self._h, ptr.ctypes.data, pts.ctypes.data,
                                      tree.ctypes.data, int(tree.size))
        if rc != 0:
            raise G.GsknnError(rc, G.last_error())

    def sync(self) -> None:
        rc = self._L.gsknn_batch_sync(self._h)
        if rc != 0:
            raise G.GsknnError(rc, G.last_error())

    def info(self) -> dict:
        ci = ctypes.c_int
        shape, rows, grid, tiles, items = ci(), ci(), ci(), ci(), ci()
        evals = ctypes.c_double()
        tune = (ctypes.c_float * 3)()
        self._L.gsknn_batch_info(self._h, ctypes.byref(shape), ctypes.byref(rows),
                                 ctypes.byref(grid), ctypes.byref(tiles), ctypes.byref(items),
                                 ctypes.byref(evals), tune)
        return {"shape": shape.value, "shape_name": SHAPES.get(shape.value, "?"),
                "tile_rows": rows.value, "grid": grid.value, "tiles": tiles.value,
                "items": items.value, "evals": evals.value,
                "tune_ms": {SHAPES[s]: round(float(tune[s]), 3) for s in range(3)
                            if tune[s] >= 0}}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.gsknn_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def forget_tuning() -> None:
    G.lib().gsknn_batch_forget_tuning()
