"""Seeded synthetic point sets for the GSKNN workloads.

All generators are built on a counter-based splitmix64 stream written in numpy, so a given
(seed, size) yields the same bits on every machine and numpy version. The point sets follow the
shapes of the reference's own drivers (test/test_dgsknn.c:121-163: a row-major N x d table,
norms precomputed per point, alpha/beta index lists) at the sizes of the benchmark workloads:

* uniform table          -- coordinates i.i.d. U[0,1)
* gaussian mixture table -- 16 isotropic Gaussians, centres U[0,1]^d, sigma 0.05
* latent-manifold table  -- U[0,1)^8 mapped into R^d by a seeded orthonormal basis, plus noise

Index arrays are int32 (the C API's `int *alpha, int *beta`).
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """n consecutive outputs of the splitmix64 generator started at `seed` (uint64)."""
    with np.errstate(over="ignore"):
        ctr = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + ctr * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, shape, offset: int = 0) -> np.ndarray:
    """float64 U[0,1) with 53 random bits."""
    n = int(np.prod(shape))
    z = splitmix64(seed, n, offset)
    return ((z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)).reshape(shape)


def normal(seed: int, shape) -> np.ndarray:
    """float64 N(0,1) by the Box-Muller transform on two uniform streams."""
    n = int(np.prod(shape))
    u1 = uniform(seed, (n,))
    u2 = uniform(seed ^ 0x5DEECE66D, (n,))
    u1 = np.maximum(u1, 1e-300)
    return (np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)).reshape(shape)


def permutation(seed: int, n: int) -> np.ndarray:
    """A seeded permutation of 0..n-1 (int64)."""
    keys = splitmix64(seed, n)
    return np.argsort(keys, kind="stable")


def randint(seed: int, n: int, high: int) -> np.ndarray:
    return (splitmix64(seed, n) % np.uint64(high)).astype(np.int64)


def sq_norms(X: np.ndarray) -> np.ndarray:
    """Squared row norms accumulated in FP64, returned in X's dtype."""
    X64 = X.astype(np.float64, copy=False)
    return np.einsum("ij,ij->i", X64, X64).astype(X.dtype)


def uniform_table(seed: int, n_points: int, d: int, dtype=np.float64) -> np.ndarray:
    return uniform(seed, (n_points, d)).astype(dtype)


def gaussian_mixture_table(seed: int, n_points: int, d: int, n_centres: int = 16,
                           sigma: float = 0.05, dtype=np.float32) -> np.ndarray:
    centres = uniform(seed + 1, (n_centres, d))
    label = randint(seed + 2, n_points, n_centres)
    X = centres[label]
    X += sigma * normal(seed + 3, (n_points, d))
    return X.astype(dtype)


def orthonormal_basis(seed: int, d: int, r: int) -> np.ndarray:
    """d x r matrix with orthonormal columns (modified Gram-Schmidt on a Gaussian matrix)."""
    G = normal(seed, (d, r))
    Q = np.zeros((d, r))
    for c in range(r):
        v = G[:, c].copy()
        for p in range(c):
            v -= np.dot(Q[:, p], v) * Q[:, p]
        Q[:, c] = v / np.linalg.norm(v)
    return Q


def latent_manifold_table(seed: int, n_points: int, d: int, latent: int = 8,
                          noise: float = 1e-3, dtype=np.float32, chunk: int = 1 << 16):
    """U[0,1)^latent mapped into R^d by a seeded orthonormal basis, plus N(0, noise^2)."""
    B = orthonormal_basis(seed + 11, d, latent)
    out = np.empty((n_points, d), dtype=dtype)
    Z = uniform(seed + 12, (n_points, latent))
    for s in range(0, n_points, chunk):
        e = min(n_points, s + chunk)
        blk = Z[s:e] @ B.T
        blk += noise * normal(seed + 13 + s, (e - s, d))
        out[s:e] = blk.astype(dtype)
    return out


class KnnProblem:
    """One fused-kNN call: table(s), norms, alpha (candidates) and beta (queries)."""

    def __init__(self, X, X2, alpha, beta, k, name=""):
        self.X = X
        self.X2 = X2
        self.alpha = np.ascontiguousarray(alpha, dtype=np.int32)
        self.beta = np.ascontiguousarray(beta, dtype=np.int32)
        self.k = int(k)
        self.name = name

    @property
    def d(self):
        return self.X.shape[1]

    @property
    def m(self):
        """Number of candidates (the C API's m)."""
        return self.alpha.size

    @property
    def n(self):
        """Number of queries = heap rows (the C API's n)."""
        return self.beta.size

    def empty_heap(self, ro=None):
        dt = self.X.dtype
        if ro is None:
            ro = np.finfo(dt).max
        D = np.full((self.n, self.k), ro, dtype=dt)
        I = np.full((self.n, self.k), -1, dtype=np.int32)
        return D, I


def config1(seed: int = 1):
    """dgsknn, float64: N=8192, d=32, U[0,1); beta (4096 queries) and alpha (4096 candidates)
    are disjoint halves of a seeded permutation; k=16. Returns (problem, alpha2) where alpha2
    is the second call's candidate list, an independent seeded draw of 4096 points."""
    N, d = 8192, 32
    X = uniform_table(seed, N, d, np.float64)
    perm = permutation(seed + 100, N)
    beta = perm[:4096]
    alpha = perm[4096:8192]
    alpha2 = permutation(seed + 200, N)[:4096]
    p = KnnProblem(X, sq_norms(X), alpha, beta, 16, "dgsknn f64 N=8192 d=32 m=n=4096 k=16")
    return p, np.ascontiguousarray(alpha2, dtype=np.int32)


def config2(seed: int = 2, n_points: int = 1 << 20, n_queries: int = 65536,
            n_refs: int = 262144, d: int = 64, k: int = 32):
    """sgsknn, float32: N=1,048,576 points of a 16-Gaussian mixture (sigma 0.05), d=64;
    65,536 queries and 262,144 references as disjoint random index subsets; k=32."""
    X = gaussian_mixture_table(seed, n_points, d, dtype=np.float32)
    perm = permutation(seed + 100, n_points)
    beta = perm[:n_queries]
    alpha = perm[n_queries:n_queries + n_refs]
    return KnnProblem(X, sq_norms(X), alpha, beta, k,
                      f"sgsknn f32 N={n_points} d={d} queries={n_queries} refs={n_refs} k={k}")


def config3(seed: int = 3, n_queries: int = 32768, n_refs: int = 262144, d: int = 256,
            k: int = 64):
    """Precision form: 32,768 queries and 262,144 references, d=256, k=64, on an 8-dim latent
    manifold (U[0,1)^8 through a seeded orthonormal basis) plus N(0, (1e-3)^2) noise."""
    N = n_queries + n_refs
    X = latent_manifold_table(seed, N, d, dtype=np.float32)
    perm = permutation(seed + 100, N)
    beta = perm[:n_queries]
    alpha = perm[n_queries:]
    return KnnProblem(X, sq_norms(X), alpha, beta, k,
                      f"precision f32 d={d} queries={n_queries} refs={n_refs} k={k}")


class AllNnProblem:
    """All-nearest-neighbour search over randomized-tree leaves (the batching form)."""

    def __init__(self, X, X2, k, trees_per_pass, passes, leaf_min, leaf_max, tree_seed, name=""):
        self.X = X
        self.X2 = X2
        self.k = int(k)
        self.trees_per_pass = int(trees_per_pass)
        self.passes = int(passes)
        self.leaf_min = int(leaf_min)
        self.leaf_max = int(leaf_max)
        self.tree_seed = int(tree_seed)
        self.name = name

    @property
    def N(self):
        return self.X.shape[0]

    @property
    def d(self):
        return self.X.shape[1]


def config4(seed: int = 4, n_points: int = 1 << 21, d: int = 64, k: int = 32,
            trees_per_pass: int = 8, passes: int = 4, leaf_min: int = 256,
            leaf_max: int = 2048):
    """Batching form: N=2,097,152 float32 points of a 16-Gaussian mixture (sigma 0.05), d=64;
    8 randomized trees per pass, leaf sizes uniform in [256, 2048], alpha = beta = leaf, k=32,
    heaps merged over 4 passes."""
    X = gaussian_mixture_table(seed, n_points, d, dtype=np.float32)
    return AllNnProblem(X, sq_norms(X), k, trees_per_pass, passes, leaf_min, leaf_max,
                        seed + 500,
                        f"all-NN over rkd-tree leaves: N={n_points} d={d} k={k} "
                        f"{trees_per_pass} trees/pass x {passes} passes, "
                        f"leaves U[{leaf_min},{leaf_max}]")
