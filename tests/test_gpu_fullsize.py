"""GPU parity against the oracle at the benchmark workloads' full sizes.

The other parity tests run the whole pipeline at up to 10,000 points, where
the oracle restates every stage in full.  Here the 500,000- and 2,000,000-
point workloads, the 1,000,000-vertex graph and instances as large as the
512-dataset workload's are checked stage by stage at their own sizes, with
the oracle restricted to what it can do in seconds: the K-Means label step
on a 100,000-point sample (the step is independent per point) chained
through exact full-size centroid updates; 2,000 co-association rows of a
500,000-point matrix (the row restatement), including rows at capacity;
the connected components of the whole graph; and whole EAC runs of
instances up to 50,000 points.
"""
import random

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

# the bench's 500k- and 2M-point workloads (n, d, mixture, k range)
WL = {
    "500k_16d": dict(n=500_000, d=16, comps=50, k=(350, 711), aniso=True, cr=20.0, sigma=1.0,
                     seed=3),
    "2m_8d": dict(n=2_000_000, d=8, comps=200, k=(700, 1401), aniso=False, cr=50.0,
                  sigma=(0.5, 3.0), seed=5),
}


@pytest.fixture(scope="module")
def T():
    import torch
    assert torch.cuda.is_available()
    return torch


def _data(cfg):
    from masters_final_b200 import workloads as W
    return W.gaussian_mixture(cfg["n"], cfg["d"], cfg["comps"], seed=cfg["seed"],
                              sigma=cfg["sigma"], center_range=cfg["cr"],
                              anisotropic=cfg["aniso"])


@pytest.mark.parametrize("name", list(WL))
def test_kmeans_partition_full_size(T, name):
    """The first partition of each workload's ensemble (same draws as the
    bench), step by step at full n: every label pass equals the oracle's on
    a 100,000-point sample (labels and float32 distances, both labelers),
    every centroid update equals the oracle's full-size update bit for bit,
    and the batched ensemble fit ends on the same labels and centroids."""
    from masters_final_b200.cluster.KMeans import kmeans_centroids, kmeans_ensemble, kmeans_label
    from masters_final_b200.utils.partition import draw_ensemble_params
    cfg = WL[name]
    x = _data(cfg)
    n = cfg["n"]
    np.random.seed(cfg["seed"])
    random.seed(cfg["seed"])
    ks, inits = draw_ensemble_params(n, list(cfg["k"]), 1)
    k = ks[0]
    X = T.from_numpy(x).cuda()
    sample = np.sort(np.random.default_rng(1).choice(n, 100_000, replace=False))
    xs = np.ascontiguousarray(x[sample])
    c = x[np.asarray(inits[0])].copy()
    for step in range(3):
        lab = {}
        for mode in ("bf16", "cuda"):
            lab[mode] = [a.cpu().numpy() for a in kmeans_label(X, T.from_numpy(c).cuda(), mode)]
        assert np.array_equal(lab["bf16"][0], lab["cuda"][0])
        assert np.array_equal(lab["bf16"][1], lab["cuda"][1])
        rl, rd = oracle.kmeans_label(xs, c)
        assert np.array_equal(lab["cuda"][0][sample], rl)
        assert np.array_equal(lab["cuda"][1][sample], rd)
        if step == 2:
            break
        labels, dists = lab["cuda"]
        g = kmeans_centroids(X, T.from_numpy(labels).cuda(), T.from_numpy(dists).cuda(), k)
        ref = oracle.kmeans_centroids(x, labels, dists, k)
        assert np.array_equal(g.cpu().numpy(), ref)
        c = ref
    Lb, Cb, _, it, _ = kmeans_ensemble(X, ks, inits, max_iter=3, label_mode="bf16")
    assert int(it[0].item()) == 3
    assert np.array_equal(Lb[0].cpu().numpy(), lab["cuda"][0])
    assert np.array_equal(Cb[0, :k].cpu().numpy(), c)


def _check_rows(T, L, n, factor, n_rows, capped_rows, seed):
    from masters_final_b200.EAC.sparse import CoassocBuilder, EAC_CSR
    b = CoassocBuilder(L, n)
    c = EAC_CSR(n, max_assocs=int(b.max_cluster * factor), condensed=True,
                max_assocs_type="linear")
    c.update_ensemble(None, builder=b)
    ip = c.indptr.cpu().numpy()
    cap = oracle.indptr_linear(n, int(b.max_cluster * factor))
    full = np.flatnonzero(np.diff(ip) == np.diff(cap))
    rng = np.random.default_rng(seed)
    rows = [rng.choice(n, n_rows, replace=False)]
    if capped_rows:
        assert c.nnz_discarded > 0 and full.size >= capped_rows
        rows.append(rng.choice(full, capped_rows, replace=False))
    rows = np.unique(np.concatenate(rows))
    Lh = L.cpu().numpy() if hasattr(L, "cpu") else L
    for i, (cols, cnt) in zip(rows, oracle.coassoc_rows(Lh, cap, rows)):
        s, e = int(ip[i]), int(ip[i + 1])
        assert np.array_equal(c.indices[s:e].cpu().numpy(), cols), i
        assert np.array_equal(c.data[s:e].cpu().numpy(), cnt), i
    return c


def test_coassoc_rows_full_size(T):
    """The 500,000-point workload's 20-partition ensemble (K-Means on the
    GPU, the default capacity factor of 3): 2,000 random rows of the matrix
    the GPU builds equal the row restatement of the reference's build."""
    from masters_final_b200.utils.partition import generate_ensemble_labels
    cfg = WL["500k_16d"]
    X = T.from_numpy(_data(cfg)).cuda()
    np.random.seed(7)
    random.seed(7)
    L, _ = generate_ensemble_labels(X, list(cfg["k"]), 20, 3, label_mode="bf16")
    _check_rows(T, L, cfg["n"], 3, 2000, 0, 11)


def test_coassoc_rows_full_size_capped(T):
    """500,000 points, 20 partitions of random labels (k about 530) and a
    capacity factor of 1: most rows hit their capacity and drop
    associations.  1,000 random rows and 1,000 rows at capacity equal the
    reference's keep-first-capacity rule, restated row by row."""
    rng = np.random.default_rng(12)
    n, P = 500_000, 20
    L = np.stack([rng.integers(0, int(rng.integers(350, 711)), n) for _ in range(P)]).astype(np.int32)
    _check_rows(T, T.from_numpy(L).cuda(), n, 1, 1000, 1000, 13)


def test_connected_components_1m_vs_oracle(T):
    """The 16-NN graph of 1,000,000 points: component labels equal the
    reference's numbering (oracle of connected_comps_seq), and a graph cut
    into pieces by dropping its heavy edges too."""
    from masters_final_b200 import workloads as W
    from masters_final_b200.graph.connected_components import connected_comps_gpu
    indptr, dest, w = W.knn_graph(1_000_000, k=16, seed=2)
    first, deg = indptr[:-1].astype(np.int32), np.diff(indptr).astype(np.int32)
    _, ref = oracle.boruvka_seq(indptr, dest, w)
    assert np.array_equal(connected_comps_gpu(dest, w, first, deg), ref)
    # keep the lightest quarter of the edges: thousands of components
    rows = np.repeat(np.arange(indptr.size - 1), np.diff(indptr))
    m = w <= 64
    ip2, d2, w2 = W.csr_from_undirected(indptr.size - 1, rows[m & (rows < dest)],
                                        dest[m & (rows < dest)].astype(np.int64),
                                        w[m & (rows < dest)])
    _, ref2 = oracle.boruvka_seq(ip2, d2, w2)
    assert np.unique(ref2).size > 1000
    got2 = connected_comps_gpu(d2, w2, ip2[:-1].astype(np.int32), np.diff(ip2).astype(np.int32))
    assert np.array_equal(got2, ref2)


BATCHED_SHAPES = [(1000, 2), (5000, 32), (20000, 8), (20000, 32), (50000, 2), (50000, 16)]


def test_batched_instances_full_size(T):
    """Instances spanning the 512-dataset workload's range (n from 1,000 to
    50,000, d from 2 to 32, 50 partitions, k from the reference's rule1) in
    one batched call: kept and discarded counts, cluster counts and final
    labels equal the oracle pipeline's."""
    import multiprocessing as mp
    from masters_final_b200 import workloads as W
    from masters_final_b200.EAC.batched import draw_instance_params, eac_batch, k_range_rule1
    xs, ps = [], []
    for i, (n, d) in enumerate(BATCHED_SHAPES):
        xs.append(W.gaussian_mixture(n, d, 3 + 4 * i, seed=100 + i, sigma=(0.5, 2.0)))
        ps.append(draw_instance_params(n, k_range_rule1(n), 50, 200 + i))
    res = eac_batch(xs, params=ps, n_workers=4)
    with mp.get_context("spawn").Pool(len(xs)) as pool:
        refs = pool.starmap(oracle.eac_pipeline, [(x, p[0], p[1], 50) for x, p in zip(xs, ps)])
    for r, (nc, labels, nnz, disc, _, _) in zip(res, refs):
        assert r.status == 0
        assert r.nnz == nnz and r.nnz_discarded == disc
        assert r.n_fclusts == max(nc, 1)
        assert np.array_equal(r.labels, labels)
