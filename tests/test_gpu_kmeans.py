"""GPU parity of K-Means labels, centroids and ensembles against the
reference's outputs and the oracle, and the end-to-end EAC pipeline."""
import random

import numpy as np
import pytest

import oracle
from tests.conftest import golden

pytestmark = pytest.mark.gpu

MODES = ["cuda", "bf16"]


@pytest.fixture(scope="module")
def T():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.mark.parametrize("mode", MODES)
def test_label_golden(T, mode):
    from masters_final_b200.cluster.KMeans import kmeans_label
    g = golden("kmeans")
    lab, d = kmeans_label(g["x"], g["c"], label_mode=mode)
    assert np.array_equal(lab.cpu().numpy(), g["labels"])
    assert np.array_equal(d.cpu().numpy(), g["dists"])


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("D,K,scale", [(1, 7, 1.0), (2, 100, 10.0), (3, 50, 1e3), (5, 130, 1.0),
                                       (8, 333, 20.0), (16, 700, 20.0), (17, 64, 5.0),
                                       (32, 257, 3.0)])
def test_label_vs_oracle(T, mode, D, K, scale):
    from masters_final_b200.cluster.KMeans import kmeans_label
    rng = np.random.default_rng(D * 1000 + K)
    x = (rng.standard_normal((20000, D)) * scale).astype(np.float32)
    c = x[rng.choice(x.shape[0], K, replace=False)].copy()
    c[K // 2] = c[K // 3]                            # duplicate centroid: exact tie
    x[:50] = c[rng.integers(0, K, 50)]               # points exactly on centroids
    lab, d = kmeans_label(x, c, label_mode=mode)
    rl, rd = oracle.kmeans_label(x, c)
    assert np.array_equal(lab.cpu().numpy(), rl)
    assert np.array_equal(d.cpu().numpy(), rd)


@pytest.mark.parametrize("mode", MODES)
def test_fit_golden(T, mode):
    from masters_final_b200.cluster.KMeans import K_Means
    g = golden("kmeans")
    random.seed(32)
    km = K_Means(n_clusters=25, max_iter=3, label_mode=mode, centroid_mode="numba")
    km.fit(g["x"])
    assert km.iters_ == g["fit_iters"]
    assert np.array_equal(km.labels_, g["fit_labels"])
    assert np.array_equal(km.cluster_centers_, g["fit_centroids"])


def test_fit_f64_centroids_and_empty_clusters(T):
    """Duplicate points as initial centroids leave a cluster empty after the
    first pass; its replacement comes from the reference's quickselect."""
    from masters_final_b200.cluster.KMeans import kmeans_ensemble
    rng = np.random.default_rng(5)
    x = rng.standard_normal((6000, 4)).astype(np.float32)
    x[1] = x[0]
    x[3] = x[2]
    inits = [[0, 1, 2, 3] + list(rng.choice(np.arange(4, 6000), 36, replace=False)),
             list(rng.choice(6000, 40, replace=False))]
    for f64 in (False, True):
        lab, cent, dist, it, inertia = kmeans_ensemble(
            x, [40, 40], inits, max_iter=4, centroid_mode="f64" if f64 else "numba")
        for p in range(2):
            rl, rc, ri = oracle.kmeans_fit(x, 40, inits[p], max_iter=4, f64=f64)
            assert np.array_equal(lab[p].cpu().numpy(), rl)
            assert np.array_equal(cent[p].cpu().numpy(), rc)
            assert int(it[p].item()) == ri


@pytest.mark.parametrize("n", [300, 1000, 2500])
def test_fit_empty_clusters_small_n(T, n):
    """Empty clusters at the batched workload's instance sizes: the range
    above the one-thread limit runs the block-parallel partition steps, which
    must reproduce the reference's selection order (three duplicated initial
    points, so three clusters empty out in the first pass)."""
    from masters_final_b200.cluster.KMeans import kmeans_ensemble
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, 3)).astype(np.float32)
    x[1], x[3], x[5] = x[0], x[2], x[4]
    k = 24
    inits = [[0, 1, 2, 3, 4, 5] + list(rng.choice(np.arange(6, n), k - 6, replace=False)),
             list(rng.choice(n, k, replace=False))]
    for f64 in (False, True):
        lab, cent, dist, it, inertia = kmeans_ensemble(
            x, [k, k], inits, max_iter=4, centroid_mode="f64" if f64 else "numba")
        for p in range(2):
            rl, rc, ri = oracle.kmeans_fit(x, k, inits[p], max_iter=4, f64=f64)
            assert np.array_equal(lab[p].cpu().numpy(), rl)
            assert np.array_equal(cent[p].cpu().numpy(), rc)
            assert int(it[p].item()) == ri


def test_fit_empty_clusters_large_n(T):
    """Empty clusters with n above the one-thread limit of the quickselect:
    the block-parallel partition steps must reproduce the reference's
    selection order exactly (ten duplicated initial points, so ten clusters
    empty out in the first pass)."""
    from masters_final_b200.cluster.KMeans import kmeans_ensemble
    rng = np.random.default_rng(12)
    n = 120_000
    x = rng.standard_normal((n, 4)).astype(np.float32)
    x[1:20:2] = x[0:20:2]
    x[5000:5010] = x[7]                  # ties among the distances as well
    inits = [list(range(20)) + list(rng.choice(np.arange(20, n), 44, replace=False)),
             list(range(0, 20, 2)) + list(range(1, 20, 2)) + list(range(20, 40))]
    ks = [64, 40]
    lab, cent, dist, it, inertia = kmeans_ensemble(x, ks, inits, max_iter=4)
    for p in range(2):
        rl, rc, ri = oracle.kmeans_fit(x, ks[p], inits[p], max_iter=4)
        assert np.array_equal(lab[p].cpu().numpy(), rl)
        assert np.array_equal(cent[p, :ks[p]].cpu().numpy(), rc)
        assert int(it[p].item()) == ri


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", ["eac_small", "eac_discard", "eac_10k"])
def test_ensemble_golden(T, mode, name):
    from masters_final_b200.utils.partition import generate_ensemble_labels
    g = golden(name)
    np.random.seed(int(g["seed"]))
    random.seed(int(g["seed"]))
    L, ks = generate_ensemble_labels(g["x"], [int(g["kmin"]), int(g["kmax"])], int(g["P"]),
                                     label_mode=mode)
    L = L.cpu().numpy()
    ref = g["labels_matrix"].astype(np.int32)
    for p in range(L.shape[0]):
        _, inv = np.unique(L[p], return_inverse=True)
        assert np.array_equal(inv, ref[p]), "partition %d" % p


@pytest.mark.parametrize("name", ["eac_small", "eac_discard", "eac_10k"])
def test_eac_end_to_end_golden(T, name):
    """Ensemble -> co-association -> Boruvka MST -> lifetime cut on the GPU:
    the final partition equals the reference's, label for label."""
    from masters_final_b200.EAC.eac import eac_pipeline
    g = golden(name)
    np.random.seed(int(g["seed"]))
    random.seed(int(g["seed"]))
    nf, labels, eac = eac_pipeline(g["x"], int(g["P"]), [int(g["kmin"]), int(g["kmax"])],
                                   factor=int(g["factor"]))
    assert eac.coassoc.nnz == g["nnz"]
    assert eac.coassoc.nnz_discarded == g["nnz_discarded"]
    assert nf == g["n_fclusts"]
    assert np.array_equal(labels, g["final_labels"])


def test_eac_drop_in_api(T):
    """The reference's call sequence: generateEnsemble, EAC(...).buildMatrix,
    finalClustering."""
    from masters_final_b200.cluster.KMeans import K_Means
    from masters_final_b200.utils.partition import generateEnsemble
    from masters_final_b200.EAC.eac import EAC
    g = golden("eac_small")
    np.random.seed(int(g["seed"]))
    random.seed(int(g["seed"]))
    ens = generateEnsemble(g["x"], K_Means(label_mode="cuda"), [int(g["kmin"]), int(g["kmax"])],
                           int(g["P"]), iters=3)
    e = EAC(g["x"].shape[0], sparse=True, condensed=True, n_partitions=int(g["P"]))
    e.buildMatrix(ens)
    assert e.sp_max_assocs == g["max_assocs"]
    labels = e.finalClustering()
    assert e.n_fclusts == g["n_fclusts"]
    assert np.array_equal(labels, g["final_labels"])
