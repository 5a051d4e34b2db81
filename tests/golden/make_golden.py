"""Generate the golden fixtures by running the reference itself.

Run where the reference sources are present, naming their root:

    EAC_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden.py

Every fixture is produced by the reference's own functions (loaded by
``refload.py``) on seeded synthetic inputs from
``masters_final_b200.workloads``; the 4elt graph is the reference's own test
fixture (tests/datasets/graphs/4elt.npz), carried here so the GPU-side tests
can use it without the reference tree.

One deliberate deviation, applied before ``finalClustering``: with SciPy >=
0.19, ``csr_matrix`` copies a data array that is a small view of a larger
buffer, so ``EAC_CSR.make_diassoc`` (MyML/MyML/EAC/sparse.py:295-304) no
longer reaches ``EAC_CSR.csr`` and Kruskal would run on raw counts.  The
reference's data flow (MyML/MyML/EAC/eac.py:128-130: condense, then diassoc,
then the MST of the diassoc matrix) is restored by pointing ``csr.data`` at
the diassoc array, as the SciPy of the reference's time did implicitly.
"""
import hashlib
import os
import random
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import refload  # noqa: E402
from masters_final_b200 import workloads as W  # noqa: E402


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def label_matrix(ensemble, n):
    """Cluster-index matrix (P x n) of a list-of-clusters ensemble."""
    L = np.full((len(ensemble), n), -1, dtype=np.int32)
    for p, part in enumerate(ensemble):
        for c, members in enumerate(part):
            L[p, members.astype(np.int64)] = c
    return L


def gen_scan(R):
    out = {}
    a = W.scan_input(100000, seed=11, hi=10000)
    o = np.empty_like(a)
    out["small_in"] = a
    out["small_total"] = np.int64(R.scan.exprefixsumNumba(a, o))
    out["small_out"] = o.copy()
    # int32 outputs wrap modulo 2^32 once the running sum passes 2^31
    b = W.scan_input(50000, seed=12, hi=200000)
    o = np.empty_like(b)
    out["wrap_in"] = b
    out["wrap_total"] = np.int64(R.scan.exprefixsumNumba(b, o))
    out["wrap_out"] = o.copy()
    c = b.astype(np.int64)
    o = np.empty_like(c)
    out["i64_total"] = np.int64(R.scan.exprefixsumNumba(c, o))
    out["i64_out"] = o.copy()
    # in-place variant with a non-zero init (exprefixsumNumbaSingle)
    d = W.scan_input(1000, seed=13, hi=50).copy()
    out["single_in"] = d.copy()
    out["single_total"] = np.int64(R.scan.exprefixsumNumbaSingle(d, 7))
    out["single_out"] = d.copy()
    np.savez_compressed(os.path.join(HERE, "scan.npz"), **out)


def boruvka_case(R, indptr, dest, w):
    first = np.ascontiguousarray(indptr[:-1], dtype=np.int32)
    deg = np.ascontiguousarray(np.diff(indptr), dtype=np.int32)
    dest = np.ascontiguousarray(dest, dtype=np.int32)
    mst, n = R.mst.boruvka_minho_seq(dest, w, first, deg)
    labels = R.cc.connected_comps_seq(dest, w, first, deg)
    mst = np.asarray(mst[:n])
    return dict(mst=mst, n_mst=np.int64(n),
                mst_weight=np.int64(w[mst].astype(np.int64).sum()),
                cc_labels=np.asarray(labels, dtype=np.int32))


def gen_graphs(R):
    import scipy.sparse as sp
    from scipy.sparse.csgraph import minimum_spanning_tree
    src = os.path.join(refload.REF, "tests/datasets/graphs/4elt.npz")
    g = np.load(src)
    indptr, dest, w = g["indptr"], g["indices"], g["data"]
    res = boruvka_case(R, indptr, dest, w)
    sm = minimum_spanning_tree(sp.csr_matrix((w, dest, indptr), shape=tuple(g["shape"])))
    res["scipy_weight"] = np.int64(sm.sum())
    res["scipy_nnz"] = np.int64(sm.nnz)
    np.savez_compressed(os.path.join(HERE, "graph_4elt.npz"), indptr=indptr,
                        indices=dest, data=w, **res)

    # kNN graph with uint8 weights and many ties, plus a disconnected graph
    ip, ind, ww = W.knn_graph(20000, k=16, seed=21)
    res = boruvka_case(R, ip, ind, ww)
    np.savez_compressed(os.path.join(HERE, "graph_knn20k.npz"), indptr=ip,
                        indices=ind, data=ww, **res)

    rng = np.random.default_rng(22)
    V = 3000
    parts = []
    for lo, hi in ((0, 1000), (1000, 1800), (1800, 2900)):   # 2900..2999 isolated
        m = (hi - lo) * 3
        a = rng.integers(lo, hi, m)
        b = rng.integers(lo, hi, m)
        keep = a != b
        parts.append((np.minimum(a, b)[keep], np.maximum(a, b)[keep]))
    a = np.concatenate([p[0] for p in parts])
    b = np.concatenate([p[1] for p in parts])
    key = np.unique(a * V + b)
    a, b = key // V, key % V
    ww = rng.integers(1, 40, a.size).astype(np.uint8)
    ip, ind, ww = W.csr_from_undirected(V, a, b, ww)
    res = boruvka_case(R, ip, ind, ww)
    np.savez_compressed(os.path.join(HERE, "graph_disconnected.npz"), indptr=ip,
                        indices=ind, data=ww, **res)


def gen_kmeans(R):
    x = W.gaussian_mixture(3000, 5, 4, seed=31)
    c = x[:40].copy()
    c[5] = 1000.0
    c[7] = -1000.0
    c[11] = c[12]            # exact tie between two centroids
    dists = np.empty(x.shape[0], dtype=np.float32)
    labels = R.kmeans.numba_label(x, c, dists, True)
    newc = R.kmeans.numba_recompute_centroids(x, c, labels, dists)
    sel = np.empty(5, dtype=np.int32)
    R.sorting.arg_k_select(dists, 5, sel)
    # one fit: 3 Lloyd iterations from a seeded random init
    random.seed(32)
    km = R.kmeans.K_Means(n_clusters=25, max_iter=3, label_mode="numba",
                          centroid_mode="numba", cuda_mem="auto")
    random.seed(32)
    init = random.sample(range(x.shape[0]), 25)
    random.seed(32)
    km.fit(x)
    np.savez_compressed(os.path.join(HERE, "kmeans.npz"), x=x, c=c, labels=labels,
                        dists=dists, new_centroids=newc, k_select=sel,
                        fit_init=np.asarray(init, dtype=np.int64),
                        fit_labels=km.labels_, fit_centroids=km.cluster_centers_,
                        fit_iters=np.int64(km.iters_))


def run_eac(R, x, P, krange, seed, factor=3):
    n = x.shape[0]
    np.random.seed(seed)
    random.seed(seed)
    gen = R.kmeans.K_Means(label_mode="numba", centroid_mode="numba", cuda_mem="auto")
    ens = R.partition.generateEnsemble(x, gen, list(krange), P, iters=3)
    e = R.eac.EAC(n, sparse=True, condensed=True, n_partitions=P,
                  sparse_max_assocs_factor=factor)
    e.buildMatrix(ens)
    counts = None
    csr = e.coassoc.csr
    if not np.shares_memory(csr.data, e.coassoc.data):
        csr.data = e.coassoc.data          # see the module docstring
    indptr = csr.indptr.astype(np.int64).copy()
    indices = csr.indices.astype(np.int32).copy()
    diassoc = csr.data.copy()
    labels = e.finalClustering()
    return dict(labels_matrix=label_matrix(ens, n), indptr=indptr, indices=indices,
                diassoc=diassoc, nnz=np.int64(e.coassoc.nnz),
                nnz_discarded=np.int64(e.coassoc.nnz_discarded),
                max_assocs=np.int64(e.sp_max_assocs),
                n_fclusts=np.int64(e.n_fclusts), final_labels=np.asarray(labels, np.int32))


def gen_eac(R):
    x = W.gaussian_mixture(1500, 2, 4, seed=41)
    r = run_eac(R, x, 30, (10, 30), seed=41)
    np.savez_compressed(os.path.join(HERE, "eac_small.npz"), x=x, P=30, kmin=10, kmax=30,
                        seed=41, factor=3, **r)
    # tight capacities: later partitions discard associations
    x = W.gaussian_mixture(2000, 2, 3, seed=42)
    r = run_eac(R, x, 25, (3, 9), seed=42, factor=1)
    assert r["nnz_discarded"] > 0, "discard case must discard"
    np.savez_compressed(os.path.join(HERE, "eac_discard.npz"), x=x, P=25, kmin=3, kmax=9,
                        seed=42, factor=1, **r)
    # the reference's CPU-runnable workload: n=10,000 2-D points, 6 Gaussians,
    # 100 partitions, k in [50, 100]
    x = W.gaussian_mixture(10000, 2, 6, seed=0)
    r = run_eac(R, x, 100, (50, 101), seed=0)
    summary = dict(x=x, P=100, kmin=50, kmax=101, seed=0, factor=3,
                   labels_matrix=r["labels_matrix"].astype(np.uint8),
                   coassoc_sha=sha(r["indptr"], r["indices"], r["diassoc"]),
                   nnz=r["nnz"], nnz_discarded=r["nnz_discarded"],
                   max_assocs=r["max_assocs"], n_fclusts=r["n_fclusts"],
                   final_labels=r["final_labels"],
                   diassoc_hist=np.bincount(r["diassoc"], minlength=256))
    np.savez_compressed(os.path.join(HERE, "eac_10k.npz"), **summary)


def gen_partition(R):
    part = np.array([1, 1, 1, 3, 2, 4, 2, 4, 3, 3], dtype=np.uint32)
    out = R.partition.convertClusterStringToIndex(part)
    np.savez(os.path.join(HERE, "partition.npz"), labels=part,
             **{"cluster%d" % i: c for i, c in enumerate(out)})


def gen_lifetime(R):
    rng = np.random.default_rng(51)
    cases = {}
    for t in range(6):
        w = np.sort(rng.integers(1, 60, rng.integers(300, 600))).astype(np.uint8)
        if t == 5:
            w[:] = 17                     # all equal: one cluster
        cont, th = R.eac.lifetime_n_clusters(w)
        cases["w%d" % t] = w
        cases["cont%d" % t] = np.int64(cont)
        cases["th%d" % t] = np.int64(th)
    np.savez_compressed(os.path.join(HERE, "lifetime.npz"), **cases)


def main():
    R = refload.load()
    gen_scan(R)
    gen_graphs(R)
    gen_kmeans(R)
    gen_partition(R)
    gen_lifetime(R)
    gen_eac(R)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
