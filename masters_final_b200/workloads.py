"""Seeded synthetic inputs for the EAC hot path.

The reference publishes no dataset for this path; these generators stand in
for it with the shapes, sizes and value distributions of the workloads the
reference's benchmarks and experiments use.  Points are emitted in random
order (not grouped by mixture component), as a real dataset would be.
"""
import numpy as np


def gaussian_mixture(n, d, n_centers, seed, sigma=1.0, center_range=10.0,
                     anisotropic=False, eig_range=(0.1, 4.0)):
    """n float32 points in d dimensions from ``n_centers`` Gaussians of equal
    weight, centres uniform in [-center_range, center_range]^d.

    ``sigma`` is a scalar or a (lo, hi) pair for a per-component standard
    deviation drawn uniformly.  ``anisotropic`` draws each component's
    covariance as Q diag(lambda) Q^T, lambda log-uniform in ``eig_range`` and Q
    a random orthogonal matrix.  Rows are shuffled.
    """
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-center_range, center_range, size=(n_centers, d))
    sizes = np.full(n_centers, n // n_centers, dtype=np.int64)
    sizes[: n - sizes.sum()] += 1
    parts = []
    for c in range(n_centers):
        m = int(sizes[c])
        z = rng.standard_normal((m, d))
        if anisotropic:
            lam = np.exp(rng.uniform(np.log(eig_range[0]), np.log(eig_range[1]), d))
            q, _ = np.linalg.qr(rng.standard_normal((d, d)))
            z = (z * np.sqrt(lam)) @ q.T
        else:
            s = sigma if np.isscalar(sigma) else rng.uniform(sigma[0], sigma[1])
            z = z * s
        parts.append(z + centers[c])
    x = np.concatenate(parts, axis=0)
    x = x[rng.permutation(n)]
    return np.ascontiguousarray(x, dtype=np.float32)


def batched_instances(m=512, seed=0, n_range=(1000, 50000), dims=(2, 4, 8, 16, 32),
                      comps=(3, 30), sigma=(0.5, 2.0), center_range=10.0):
    """The batched EAC workload: ``m`` independent datasets, n log-uniform in
    ``n_range``, d uniform over ``dims``, a number of Gaussians uniform in
    [comps[0], comps[1]] with per-component sigma uniform in ``sigma`` and
    centres uniform in [-center_range, center_range]^d."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(m):
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        d = int(rng.choice(dims))
        c = int(rng.integers(comps[0], comps[1] + 1))
        out.append(gaussian_mixture(n, d, c, seed=int(rng.integers(1 << 31)), sigma=sigma,
                                    center_range=center_range))
    return out


def knn_graph(n_vertices, k=16, dim=3, seed=2, wmax=255, wdtype=np.uint8):
    """Symmetric CSR graph of the k nearest neighbours of uniform points in
    [0,1)^dim: every kNN pair becomes one undirected edge (duplicates merged)
    whose integer weight is uniform in [1, wmax]; both directions are stored,
    rows sorted by column.  Returns (indptr int64, indices int32, weights)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    pts = rng.random((n_vertices, dim))
    _, nbr = cKDTree(pts).query(pts, k=k + 1, workers=-1)
    u = np.repeat(np.arange(n_vertices, dtype=np.int64), k)
    v = nbr[:, 1:].reshape(-1).astype(np.int64)
    a, b = np.minimum(u, v), np.maximum(u, v)
    key = np.unique(a * n_vertices + b)
    a, b = key // n_vertices, key % n_vertices
    w = rng.integers(1, wmax + 1, size=key.size).astype(wdtype)
    return csr_from_undirected(n_vertices, a, b, w)


def csr_from_undirected(n_vertices, a, b, w):
    """Symmetric CSR (indptr int64, indices int32, weights) of undirected
    edges (a, b, w), both directions stored, rows sorted by column."""
    src = np.concatenate([a, b])
    dst = np.concatenate([b, a])
    ww = np.concatenate([w, w])
    order = np.lexsort((dst, src))
    src, dst, ww = src[order], dst[order], ww[order]
    indptr = np.zeros(n_vertices + 1, dtype=np.int64)
    np.cumsum(np.bincount(src, minlength=n_vertices), out=indptr[1:])
    return indptr, dst.astype(np.int32), ww


def scan_input(n, seed=3, hi=1000):
    """int32 values uniform in [0, hi]."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, hi + 1, size=n, dtype=np.int32)
