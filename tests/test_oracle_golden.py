"""The oracle against the reference's own outputs (fixtures made by running
the reference, tests/golden/make_golden.py) and its known-answer tests."""
import numpy as np
import pytest

import oracle
from tests.conftest import golden


def test_scan_small():
    g = golden("scan")
    out, tot = oracle.exprefixsum(g["small_in"])
    assert tot == g["small_total"]
    assert np.array_equal(out, g["small_out"])


def test_scan_wraps_int32_like_reference():
    g = golden("scan")
    out, tot = oracle.exprefixsum(g["wrap_in"])
    assert tot == g["wrap_total"] and tot > 2 ** 31
    assert np.array_equal(out, g["wrap_out"])
    out64, tot64 = oracle.exprefixsum(g["wrap_in"].astype(np.int64))
    assert np.array_equal(out64, g["i64_out"]) and tot64 == g["i64_total"]


def test_scan_init():
    g = golden("scan")
    out, tot = oracle.exprefixsum(g["single_in"], init=7)
    assert tot == g["single_total"]
    assert np.array_equal(out, g["single_out"])


@pytest.mark.parametrize("name", ["graph_4elt", "graph_knn20k", "graph_disconnected"])
def test_boruvka_seq_matches_reference(name):
    g = golden(name)
    mst, labels = oracle.boruvka_seq(g["indptr"], g["indices"], g["data"])
    assert np.array_equal(mst, g["mst"])
    assert np.array_equal(labels, g["cc_labels"])


def test_4elt_known_answer():
    # tests/MyML/test_boruvka.py:130-159: edge count and total weight = SciPy's
    g = golden("graph_4elt")
    assert g["n_mst"] == g["scipy_nnz"] == 15605
    assert g["mst_weight"] == g["scipy_weight"] == 2964801


@pytest.mark.parametrize("name", ["graph_4elt", "graph_knn20k", "graph_disconnected"])
def test_kruskal_tiebreak_forest_has_reference_weight(name):
    g = golden(name)
    a, b, w = oracle.upper_edges(g["indptr"], g["indices"], g["data"])
    f = oracle.kruskal_forest(g["indptr"].size - 1, a, b, w)
    assert f.sum() == g["n_mst"]
    assert w[f].astype(np.int64).sum() == g["mst_weight"]


def test_kmeans_label_and_centroids():
    g = golden("kmeans")
    lab, d = oracle.kmeans_label(g["x"], g["c"])
    assert np.array_equal(lab, g["labels"])
    assert np.array_equal(d, g["dists"])
    newc = oracle.kmeans_centroids(g["x"], lab, d, g["c"].shape[0])
    assert np.array_equal(newc, g["new_centroids"])
    assert np.array_equal(oracle.arg_k_select(d, 5), g["k_select"])


def test_kmeans_fit():
    g = golden("kmeans")
    lab, c, it = oracle.kmeans_fit(g["x"], 25, g["fit_init"], max_iter=3)
    assert it == g["fit_iters"]
    assert np.array_equal(lab, g["fit_labels"])
    assert np.array_equal(c, g["fit_centroids"])


def test_np_sum_emulation():
    rng = np.random.default_rng(0)
    for n in (1, 7, 8, 127, 128, 129, 1000, 8193, 100003):
        a = (rng.random(n) * 1000).astype(np.float32)
        assert oracle.np_sum_f32(a) == a.sum()


def test_partition_known_answer():
    # tests/MyML/utils/test_partition.py:81-97
    g = golden("partition")
    lab = g["labels"]
    _, inv = np.unique(lab, return_inverse=True)
    for c in range(4):
        assert np.array_equal(np.nonzero(inv == c)[0].astype(np.uint64), g["cluster%d" % c])


def test_lifetime():
    g = golden("lifetime")
    for t in range(6):
        cont, th = oracle.lifetime_n_clusters(g["w%d" % t])
        assert cont == g["cont%d" % t] and th == g["th%d" % t]


@pytest.mark.parametrize("name", ["eac_small", "eac_discard"])
def test_eac_pipeline(name):
    g = golden(name)
    x = g["x"]
    n = x.shape[0]
    np.random.seed(int(g["seed"]))
    import random
    random.seed(int(g["seed"]))
    params = oracle.draw_ensemble_params(n, [int(g["kmin"]), int(g["kmax"])], int(g["P"]))
    L = oracle.ensemble_labels(x, params)
    assert np.array_equal(L, g["labels_matrix"])
    ma = oracle.max_cluster_size(L) * int(g["factor"])
    assert ma == g["max_assocs"]
    ip, ind, cnt, nnz, disc, st = oracle.coassoc_build(L, oracle.indptr_linear(n, ma))
    assert st == 0
    assert nnz == g["nnz"] and disc == g["nnz_discarded"]
    dia = (cnt.max() + 1 - cnt).astype(np.uint8)
    assert np.array_equal(ip, g["indptr"])
    assert np.array_equal(ind, g["indices"])
    assert np.array_equal(dia, g["diassoc"])
    rows = np.repeat(np.arange(n), np.diff(ip))
    nc, lab = oracle.sp_sl_lifetime(n, rows, ind.astype(np.int64), dia, int(g["P"]))
    assert nc == g["n_fclusts"]
    assert np.array_equal(lab, g["final_labels"])


@pytest.mark.parametrize("name", ["eac_small", "eac_discard", "eac_10k"])
def test_coassoc_rows_match_reference(name):
    """The row-by-row restatement of the co-association build (used to check
    sampled rows of matrices too large for the full restatement) gives the
    reference's own rows, including rows that hit their capacity."""
    g = golden(name)
    L = g["labels_matrix"]
    n = L.shape[1]
    cap = oracle.indptr_linear(n, int(g["max_assocs"]))
    if "indptr" in g:
        ip, ind, dia = g["indptr"], g["indices"], g["diassoc"]
    else:
        # the 10k fixture keeps a digest of its matrix, which
        # test_coassoc_10k_digest pins the full restatement to
        ip, ind, cnt, _, _, _ = oracle.coassoc_build(L, cap)
        dia = (cnt.max() + 1 - cnt).astype(np.uint8)
    full = np.flatnonzero(np.diff(ip) == np.diff(cap))          # rows at capacity
    rng = np.random.default_rng(5)
    rows = np.unique(np.concatenate([rng.choice(n, min(n, 300), replace=False), full[:300]]))
    const = None
    for i, (cols, cnt) in zip(rows, oracle.coassoc_rows(L, cap, rows)):
        s, e = ip[i], ip[i + 1]
        assert np.array_equal(cols, ind[s:e])
        tot = cnt.astype(np.int64) + dia[s:e].astype(np.int64)    # diassoc = max + 1 - count
        if tot.size:
            const = tot[0] if const is None else const
            assert np.all(tot == const)
    if name == "eac_discard":
        assert full.size > 0


def test_coassoc_10k_digest():
    """The full restatement reproduces the reference's 10k-point matrix
    (indptr, indices and dissimilarities, by digest) and counts."""
    import hashlib
    g = golden("eac_10k")
    L = g["labels_matrix"]
    n = L.shape[1]
    ip, ind, cnt, nnz, disc, st = oracle.coassoc_build(L, oracle.indptr_linear(n, int(g["max_assocs"])))
    assert st == 0 and nnz == g["nnz"] and disc == g["nnz_discarded"]
    dia = (cnt.max() + 1 - cnt).astype(np.uint8)
    h = hashlib.sha256()
    for a in (ip, ind, dia):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == str(g["coassoc_sha"])
