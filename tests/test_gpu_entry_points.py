"""GPU parity of the single-step entry points (fixed-mode label steps, one
centroid update, the one-call co-association build, the lifetime cut and
the canonical relabelling) against the oracle and the reference's outputs."""
import ctypes

import numpy as np
import pytest

import oracle
from tests.conftest import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    import torch
    assert torch.cuda.is_available()
    return torch


def _ws(T, nbytes):
    return T.empty(max(int(nbytes), 256), dtype=T.uint8, device="cuda")


@pytest.mark.parametrize("fn", ["eacb_kmeans_label_fp32", "eacb_kmeans_label_bf16tc"])
def test_label_fixed_modes(T, fn):
    from masters_final_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(4)
    x = (rng.standard_normal((30000, 12)) * 4).astype(np.float32)
    c = x[rng.choice(30000, 150, replace=False)].copy()
    c[7] = c[3]
    xd, cd = T.from_numpy(x).cuda(), T.from_numpy(c).cuda()
    lab = T.empty(30000, dtype=T.int32, device="cuda")
    dist = T.empty(30000, dtype=T.float32, device="cuda")
    ws = _ws(T, L.eacb_kmeans_label_workspace_size(30000, 12, 150))
    _lib.check(getattr(L, fn)(_lib.ptr(xd), 30000, 12, _lib.ptr(cd), 150, _lib.ptr(lab),
                              _lib.ptr(dist), _lib.ptr(ws), ws.numel(), None), fn)
    rl, rd = oracle.kmeans_label(x, c)
    assert np.array_equal(lab.cpu().numpy(), rl)
    assert np.array_equal(dist.cpu().numpy(), rd)


@pytest.mark.parametrize("f64", [False, True])
def test_centroid_update_with_empty_clusters(T, f64):
    """Duplicate centroids leave clusters empty; n is above the one-thread
    limit of the quickselect that refills them."""
    from masters_final_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(9)
    n, d, k = 50000, 6, 90
    x = rng.standard_normal((n, d)).astype(np.float32)
    c = x[rng.choice(n, k, replace=False)].copy()
    c[10:20] = c[0:10]                        # ten duplicates: ten empty clusters
    labels, dists = oracle.kmeans_label(x, c)
    xd = T.from_numpy(x).cuda()
    ld = T.from_numpy(labels.astype(np.int32)).cuda()
    dd = T.from_numpy(dists.copy()).cuda()
    out = T.zeros((k, d), dtype=T.float32, device="cuda")
    ws = _ws(T, L.eacb_kmeans_centroids_workspace_size(n, d, k))
    _lib.check(L.eacb_kmeans_centroids(_lib.ptr(xd), n, d, _lib.ptr(ld), _lib.ptr(dd), k,
                                       1 if f64 else 0, _lib.ptr(out), _lib.ptr(ws), ws.numel(),
                                       None), "centroids")
    ref = oracle.kmeans_centroids(x, labels, dists.copy(), k, f64=f64)
    assert np.array_equal(out.cpu().numpy(), ref)
    assert np.array_equal(dd.cpu().numpy(), dists)          # distances left unchanged


@pytest.mark.parametrize("name", ["eac_small", "eac_discard"])
def test_coassoc_build_one_call(T, name):
    from masters_final_b200 import _lib
    L = _lib.load()
    g = golden(name)
    lm = g["labels_matrix"].astype(np.int32)
    P, n = lm.shape
    K = int(lm.max()) + 1
    labels = T.from_numpy(lm).cuda()
    ma = oracle.max_cluster_size(lm) * int(g["factor"])
    cap_total = int(oracle.indptr_linear(n, ma)[-1])
    indptr = T.empty(n + 1, dtype=T.int64, device="cuda")
    ind = T.empty(cap_total, dtype=T.int32, device="cuda")
    dat = T.empty(cap_total, dtype=T.uint8, device="cuda")
    nnz, disc, mx, mao = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int64()
    ws = _ws(T, L.eacb_coassoc_build_workspace_size(n, P, K))
    _lib.check(L.eacb_coassoc_build(_lib.ptr(labels), n, P, K, 0, 0, int(g["factor"]),
                                    _lib.ptr(indptr), _lib.ptr(ind), _lib.ptr(dat), cap_total, 1,
                                    ctypes.byref(nnz), ctypes.byref(disc), ctypes.byref(mx),
                                    ctypes.byref(mao), _lib.ptr(ws), ws.numel(), None), "build")
    assert mao.value == g["max_assocs"]
    assert nnz.value == g["nnz"] and disc.value == g["nnz_discarded"]
    assert np.array_equal(indptr.cpu().numpy(), g["indptr"])
    assert np.array_equal(ind[:nnz.value].cpu().numpy(), g["indices"])
    assert np.array_equal(dat[:nnz.value].cpu().numpy(), g["diassoc"])


def _cut(T, L, _lib, w, n, max_dist, n_clusters=0):
    wd = T.from_numpy(np.ascontiguousarray(w, dtype=np.uint8)).cuda()
    nc, th = ctypes.c_int64(), ctypes.c_int32()
    ws = _ws(T, L.eacb_lifetime_cut_workspace_size())
    st = L.eacb_lifetime_cut(_lib.ptr(wd), int(w.size), n, max_dist, n_clusters,
                             ctypes.byref(nc), ctypes.byref(th), _lib.ptr(ws), ws.numel(), None)
    return st, nc.value, th.value


def test_lifetime_cut(T):
    from masters_final_b200 import _lib
    L = _lib.load()
    for name in ("eac_small", "eac_discard"):
        g = golden(name)
        n = g["x"].shape[0]
        ip, idx, w = g["indptr"], g["indices"], g["diassoc"]
        a = np.repeat(np.arange(n), np.diff(ip))
        f = oracle.kruskal_forest(n, a, idx.astype(np.int64), w)
        rng = np.random.default_rng(1)
        fw = w[f][rng.permutation(int(f.sum()))]          # any order
        st, nc, th = _cut(T, L, _lib, fw, n, int(g["P"]))
        assert st == 0 and nc == g["n_fclusts"]
        exp_nc, _ = oracle.sp_sl_lifetime(n, a, idx.astype(np.int64), w, int(g["P"]))
        assert nc == exp_nc
    st, _, _ = _cut(T, L, _lib, np.array([3], dtype=np.uint8), 10, 5)
    assert st == _lib.ERR_VALUE                                # fewer than two forest edges


def test_relabel_canonical(T):
    from masters_final_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(2)
    n = 300_000
    lab = rng.integers(0, 5000, n).astype(np.int32)
    ld = T.from_numpy(lab).cuda()
    out = T.empty_like(ld)
    ng = ctypes.c_int64()
    ws = _ws(T, L.eacb_relabel_canonical_workspace_size(n))
    _lib.check(L.eacb_relabel_canonical(_lib.ptr(ld), n, _lib.ptr(out), ctypes.byref(ng),
                                        _lib.ptr(ws), ws.numel(), None), "relabel")
    assert np.array_equal(out.cpu().numpy(), oracle.canonical_labels(lab))
    assert ng.value == np.unique(lab).size
    bad = ld.clone()
    bad[5] = n
    assert L.eacb_relabel_canonical(_lib.ptr(bad), n, _lib.ptr(out), ctypes.byref(ng),
                                    _lib.ptr(ws), ws.numel(), None) == -8


def test_python_step_wrappers(T):
    """The Python entry points over the same calls."""
    from masters_final_b200.cluster.KMeans import kmeans_centroids
    from masters_final_b200.EAC.eac import lifetime_cut_gpu, relabel_canonical
    rng = np.random.default_rng(6)
    x = rng.standard_normal((4000, 3)).astype(np.float32)
    c = x[:25].copy()
    c[5] = c[4]
    lab, dist = oracle.kmeans_label(x, c)
    C = kmeans_centroids(x, lab, dist, 25)
    assert np.array_equal(C.cpu().numpy(), oracle.kmeans_centroids(x, lab, dist.copy(), 25))
    g = golden("eac_small")
    n = g["x"].shape[0]
    a = np.repeat(np.arange(n), np.diff(g["indptr"]))
    f = oracle.kruskal_forest(n, a, g["indices"].astype(np.int64), g["diassoc"])
    nc, th = lifetime_cut_gpu(g["diassoc"][f], n, int(g["P"]))
    assert nc == g["n_fclusts"]
    with pytest.raises(ValueError):
        lifetime_cut_gpu(np.array([1], dtype=np.uint8), 10, 5)
    out, ng = relabel_canonical(g["final_labels"][::-1].copy())
    assert np.array_equal(out.cpu().numpy(), oracle.canonical_labels(g["final_labels"][::-1]))


def test_misaligned_workspace_refused(T):
    """A workspace that is not 256-byte aligned is refused before any launch."""
    from masters_final_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(4)
    x = rng.standard_normal((1000, 4)).astype(np.float32)
    xd = T.from_numpy(x).cuda()
    cd = xd[:10].clone()
    lab = T.empty(1000, dtype=T.int32, device="cuda")
    dist = T.empty(1000, dtype=T.float32, device="cuda")
    nb = L.eacb_kmeans_label_workspace_size(1000, 4, 10)
    ws = _ws(T, nb + 512)
    st = L.eacb_kmeans_label_fp32(_lib.ptr(xd), 1000, 4, _lib.ptr(cd), 10, _lib.ptr(lab),
                                  _lib.ptr(dist), ctypes.c_void_p(ws.data_ptr() + 16),
                                  ws.numel() - 16, None)
    assert st == _lib.ERR_WORKSPACE
    _lib.check(L.eacb_kmeans_label_fp32(_lib.ptr(xd), 1000, 4, _lib.ptr(cd), 10, _lib.ptr(lab),
                                        _lib.ptr(dist), _lib.ptr(ws), ws.numel(), None), "label")
