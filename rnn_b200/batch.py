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
          2: "64-row tiles, 4x4 per thread", 3: "tensor cores, split BF16 + FP64 re-rank"}


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
        tune = (ctypes.c_float * 4)()
        self._L.gsknn_batch_info(self._h, ctypes.byref(shape), ctypes.byref(rows),
                                 ctypes.byref(grid), ctypes.byref(tiles), ctypes.byref(items),
                                 ctypes.byref(evals), tune)
        return {"shape": shape.value, "shape_name": SHAPES.get(shape.value, "?"),
                "tile_rows": rows.value, "grid": grid.value, "tiles": tiles.value,
                "items": items.value, "evals": evals.value,
                "tune_ms": {SHAPES[s]: round(float(tune[s]), 3) for s in range(4)
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


class StreamJob:
    """The batching form with the point table and the heaps in HOST memory
    (`gsknn_stream_create`): numpy arrays X (float32 N x d), X2 (float32 N), D (float32
    N x ldD), I (int32 N x ldD), or the arrays of a mapped `Table`. Every pass streams groups of
    whole leaves (at most `group_points` points) through a device staging table and updates D / I
    in place; the results equal a resident `BatchJob`'s after the same passes."""

    def __init__(self, X, X2, D, I, k: int, group_points: int, leaf_min: int, shape: int = -1):
        for a, dt in ((X, np.float32), (X2, np.float32), (D, np.float32), (I, np.int32)):
            assert a.dtype == dt and a.flags["C_CONTIGUOUS"]
        self._keep = (X, X2, D, I)
        N, d = X.shape
        self.N, self.d, self.k = N, d, k
        L = G.lib()
        vp, ci = ctypes.c_void_p, ctypes.c_int
        L.gsknn_stream_create.restype = vp
        L.gsknn_stream_create.argtypes = [ci, ci, ci, vp, vp, vp, vp, ci, ci, ci, ci]
        L.gsknn_stream_pass.argtypes = [vp, vp, vp, vp, ci]
        L.gsknn_stream_info.argtypes = [vp] + [vp] * 4
        L.gsknn_stream_destroy.argtypes = [vp]
        self._L = L
        h = L.gsknn_stream_create(N, d, k, X.ctypes.data, X2.ctypes.data, D.ctypes.data,
                                  I.ctypes.data, D.shape[1], group_points, leaf_min, shape)
        if not h:
            raise G.GsknnError(L.gsknn_last_error(), G.last_error())
        self._h = h

    def run_pass(self, leaves: Leaves) -> None:
        """One pass over these leaves; returns when the host heaps are updated."""
        ptr = np.ascontiguousarray(leaves.ptr, dtype=np.int32)
        pts = np.ascontiguousarray(leaves.pts, dtype=np.int32)
        tree = np.ascontiguousarray(leaves.tree, dtype=np.int32)
        rc = self._L.gsknn_stream_pass(self._h, ptr.ctypes.data, pts.ctypes.data,
                                       tree.ctypes.data, int(tree.size))
        if rc != 0:
            raise G.GsknnError(rc, G.last_error())

    def info(self) -> dict:
        groups = ctypes.c_int()
        h2d, d2h, ms = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._L.gsknn_stream_info(self._h, ctypes.byref(groups), ctypes.byref(h2d),
                                  ctypes.byref(d2h), ctypes.byref(ms))
        return {"groups": groups.value, "h2d_bytes": h2d.value, "d2h_bytes": d2h.value,
                "pass_ms": ms.value}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.gsknn_stream_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_table(path: str, X: np.ndarray, X2: np.ndarray | None = None) -> None:
    """Write the N x d float32 table X (and its squared norms, computed when X2 is None) in the
    on-disk point-table format (`gsknn_table_write`)."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    L = G.lib()
    L.gsknn_table_write.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_longlong, ctypes.c_int]
    x2 = None if X2 is None else np.ascontiguousarray(X2, dtype=np.float32)
    rc = L.gsknn_table_write(path.encode(), X.ctypes.data,
                             None if x2 is None else x2.ctypes.data, X.shape[0], X.shape[1])
    if rc != 0:
        raise G.GsknnError(rc, G.last_error())


class Table:
    """A point table mapped read-only from disk (`gsknn_table_open`); `X` and `X2` are numpy
    views of the mapping, valid until `close`."""

    def __init__(self, path: str):
        L = G.lib()
        vp = ctypes.c_void_p
        L.gsknn_table_open.restype = vp
        L.gsknn_table_open.argtypes = [ctypes.c_char_p]
        for nm in ("gsknn_table_rows", "gsknn_table_dim", "gsknn_table_points",
                   "gsknn_table_norms", "gsknn_table_close"):
            getattr(L, nm).argtypes = [vp]
        L.gsknn_table_rows.restype = ctypes.c_longlong
        L.gsknn_table_points.restype = ctypes.POINTER(ctypes.c_float)
        L.gsknn_table_norms.restype = ctypes.POINTER(ctypes.c_float)
        self._L = L
        h = L.gsknn_table_open(path.encode())
        if not h:
            raise G.GsknnError(L.gsknn_last_error(), G.last_error())
        self._h = h
        self.N, self.d = int(L.gsknn_table_rows(h)), int(L.gsknn_table_dim(h))
        self.X = np.ctypeslib.as_array(L.gsknn_table_points(h), shape=(self.N, self.d))
        self.X2 = np.ctypeslib.as_array(L.gsknn_table_norms(h), shape=(self.N,))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.X = self.X2 = None
            self._L.gsknn_table_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
