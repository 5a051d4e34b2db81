"""GPU parity: scan, Boruvka MST, connected components and the EAC final
clustering against the oracle and the reference's golden outputs."""
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


def test_scan_golden(T):
    from masters_final_b200.utils.scan import exprefixsumNumba, scan_gpu, exprefixsumNumbaSingle
    g = golden("scan")
    out = np.empty_like(g["small_in"])
    assert exprefixsumNumba(g["small_in"], out) == g["small_total"]
    assert np.array_equal(out, g["small_out"])
    out = np.empty_like(g["wrap_in"])
    assert exprefixsumNumba(g["wrap_in"], out) == g["wrap_total"]
    assert np.array_equal(out, g["wrap_out"])
    a64 = g["wrap_in"].astype(np.int64)
    out = np.empty_like(a64)
    assert exprefixsumNumba(a64, out) == g["i64_total"]
    assert np.array_equal(out, g["i64_out"])
    d = g["single_in"].copy()
    assert exprefixsumNumbaSingle(d, 7) == g["single_total"]
    assert np.array_equal(d, g["single_out"])
    x = g["small_in"].copy()
    assert scan_gpu(x) == g["small_total"]
    assert np.array_equal(x, g["small_out"])


@pytest.mark.parametrize("n", [0, 1, 2, 31, 4095, 4096, 4097, 2048 * 3 + 5, 1 << 20, 3_000_001])
def test_scan_sizes(T, n):
    from masters_final_b200.utils.scan import exprefixsumNumba
    rng = np.random.default_rng(n)
    a = rng.integers(-1000, 100000, n).astype(np.int32)
    out = np.empty_like(a)
    tot = exprefixsumNumba(a, out, init=3)
    ref, rt = oracle.exprefixsum(a, init=3)
    assert tot == rt
    assert np.array_equal(out, ref)


def test_scan_64m_device_property(T):
    """The full-size stream (64 Mi int32 uniform in [0, 1000]) on device:
    differences of the output give back the input, and the total is exact."""
    from masters_final_b200 import workloads as W
    from masters_final_b200.utils.scan import scan_gpu
    a = W.scan_input(64 << 20, seed=3)
    d = T.from_numpy(a).cuda()
    x = d.clone()
    tot = scan_gpu(x)
    assert int(tot.item()) == int(a.astype(np.int64).sum())
    assert T.equal((x[1:] - x[:-1]), d[:-1])
    assert int(x[0].item()) == 0


def _check_mst(indptr, dest, w, mst, n):
    V = indptr.size - 1
    rows = np.repeat(np.arange(V), np.diff(indptr))
    a, b = rows[mst[:n]], dest[mst[:n]]
    assert np.all(a < b)
    ua, ub, uw = oracle.upper_edges(indptr, dest, w)
    f = oracle.kruskal_forest(V, ua, ub, uw)
    got = set(zip(a.tolist(), b.tolist()))
    exp = set(zip(ua[f].tolist(), ub[f].tolist()))
    assert got == exp
    return w[mst[:n]].astype(np.int64).sum()


@pytest.mark.parametrize("name", ["graph_4elt", "graph_knn20k", "graph_disconnected"])
def test_boruvka_golden(T, name):
    from masters_final_b200.graph.mst import boruvka_minho_gpu
    g = golden(name)
    indptr, dest, w = g["indptr"], g["indices"], g["data"]
    first = indptr[:-1].astype(np.int32)
    deg = np.diff(indptr).astype(np.int32)
    mst, n = boruvka_minho_gpu(dest, w, first, deg)
    assert n == g["n_mst"]
    assert _check_mst(indptr, dest, w, mst, n) == g["mst_weight"]


@pytest.mark.parametrize("name", ["graph_4elt", "graph_knn20k", "graph_disconnected"])
def test_connected_components_golden(T, name):
    from masters_final_b200.graph.connected_components import connected_comps_gpu
    g = golden(name)
    indptr, dest, w = g["indptr"], g["indices"], g["data"]
    labels = connected_comps_gpu(dest, w, indptr[:-1].astype(np.int32),
                                 np.diff(indptr).astype(np.int32))
    assert np.array_equal(labels, g["cc_labels"])


def test_boruvka_knn_1m_properties(T):
    """The full-size graph (1M points, 16-NN, uint8 weights): the forest is
    exactly the oracle Kruskal forest under (w, min, max)."""
    from masters_final_b200 import workloads as W
    from masters_final_b200.graph.mst import boruvka_minho_gpu
    indptr, dest, w = W.knn_graph(1_000_000, k=16, seed=2)
    mst, n = boruvka_minho_gpu(dest, w, indptr[:-1].astype(np.int32),
                               np.diff(indptr).astype(np.int32))
    assert n == 999_999
    _check_mst(indptr, dest, w, mst, n)


@pytest.mark.parametrize("n,k,seed", [(200_000, 8, 11), (3000, 4, 12)])
def test_round_team_sizes_agree(T, n, k, seed):
    """The round kernel runs as one block or as a cooperative grid of any
    size; the forest (as a set and in its emitted order) and the component
    labels do not depend on it, and profiling (which times each launch and
    reads the round sizes back) changes nothing."""
    from masters_final_b200 import _lib, workloads as W
    from masters_final_b200.graph.mst import boruvka_minho_gpu
    from masters_final_b200.graph.connected_components import connected_comps_gpu
    indptr, dest, w = W.knn_graph(n, k=k, seed=seed)
    first, deg = indptr[:-1].astype(np.int32), np.diff(indptr).astype(np.int32)
    L = _lib.load()
    runs = []
    try:
        for team, prof in ((0, False), (1, False), (2, False), (7, True), (1000, False)):
            L.eacb_debug_set_round_team(team)
            _lib.profile_enable(prof)
            mst, nm = boruvka_minho_gpu(dest, w, first, deg)
            cc = connected_comps_gpu(dest, w, first, deg)
            if prof:
                _, ms, _, cnt = _lib.profile_read()
                assert cnt[0] > 0 and ms[0] > 0          # round kernels were timed
            _lib.profile_enable(False)
            runs.append((mst[:nm].copy(), cc))
    finally:
        L.eacb_debug_set_round_team(0)
        _lib.profile_enable(False)
    for mst, cc in runs[1:]:
        assert np.array_equal(mst, runs[0][0])
        assert np.array_equal(cc, runs[0][1])
    _check_mst(indptr, dest, w, runs[0][0], runs[0][0].size)
    _, ref = oracle.boruvka_seq(indptr, dest, w)
    assert np.array_equal(runs[0][1], ref)


@pytest.mark.parametrize("dt", [np.uint16, np.int32, np.float32])
def test_boruvka_weight_types(T, dt):
    from masters_final_b200 import workloads as W
    from masters_final_b200.graph.mst import boruvka_minho_gpu
    rng = np.random.default_rng(7)
    indptr, dest, w8 = W.knn_graph(3000, k=8, seed=5)
    ua, ub, _ = oracle.upper_edges(indptr, dest, w8)
    if dt == np.float32:
        uw = rng.standard_normal(ua.size).astype(np.float32)
    else:
        uw = rng.integers(0 if dt == np.uint16 else -50, 50, ua.size).astype(dt)
    ip, d, w = W.csr_from_undirected(3000, ua, ub, uw)
    mst, n = boruvka_minho_gpu(d, w, ip[:-1].astype(np.int32), np.diff(ip).astype(np.int32))
    f = oracle.kruskal_forest(3000, ua, ub, uw)
    assert n == f.sum()
    _check_mst(ip, d, w, mst, n)


def _layout_permuted(indptr, dest, w, seed):
    """The same rows stored in a random order, 0-2 junk entries before each
    (first / deg point at each row's new place): no warp of 32 consecutive
    vertices finds its rows back to back."""
    V = indptr.size - 1
    rng = np.random.default_rng(seed)
    order = rng.permutation(V)
    deg = np.diff(indptr).astype(np.int32)
    gaps = rng.integers(0, 3, V)
    starts = np.concatenate([[0], np.cumsum(deg[order] + gaps)])
    d2 = np.zeros(int(starts[-1]), np.int32)
    w2 = np.full(int(starts[-1]), 255, w.dtype)
    first = np.empty(V, np.int32)
    for pos, u in enumerate(order):
        f = int(starts[pos] + gaps[pos])
        first[u] = f
        d2[f:f + deg[u]] = dest[indptr[u]:indptr[u + 1]]
        w2[f:f + deg[u]] = w[indptr[u]:indptr[u + 1]]
    return first, deg, d2, w2


def _with_parallel(indptr, dest, w, seed):
    """5% of the undirected edges get a second entry at the end of both
    rows: half with the same weight (the first entry stays the one an MST
    returns), half one lighter (the new entry becomes it)."""
    V = indptr.size - 1
    rng = np.random.default_rng(seed)
    ua, ub, uw = oracle.upper_edges(indptr, dest, w)
    pick = rng.choice(ua.size, ua.size // 20, replace=False)
    rows = [list(zip(dest[indptr[u]:indptr[u + 1]].tolist(), w[indptr[u]:indptr[u + 1]].tolist()))
            for u in range(V)]
    for j, i in enumerate(pick):
        a, b, x = int(ua[i]), int(ub[i]), int(uw[i])
        x2 = x if (j % 2 == 0 or x == 0) else x - 1
        rows[a].append((b, x2))
        rows[b].append((a, x2))
    deg = np.array([len(r) for r in rows], np.int32)
    ip = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    d2 = np.array([e[0] for r in rows for e in r], np.int32)
    w2 = np.array([e[1] for r in rows for e in r], w.dtype)
    return ip[:-1].astype(np.int32), deg, d2, w2


def _check_layout(first, deg, dest, w, mst, n):
    """MST ids on any row layout: each is the first entry of row min(u,v)
    with its destination and weight, and the forest (as pairs, and its total
    weight) is the oracle Kruskal forest.  Returns the canonical CSR."""
    V = first.size
    rows = np.full(dest.size, -1, np.int64)
    for u in range(V):
        rows[first[u]:first[u] + deg[u]] = u
    ids = mst[:n].astype(np.int64)
    a, b = rows[ids], dest[ids].astype(np.int64)
    assert np.all(a >= 0) and np.all(a < b)
    for e, u, v in zip(ids.tolist(), a.tolist(), b.tolist()):
        seg = slice(int(first[u]), e)
        assert not np.any((dest[seg] == v) & (w[seg] == w[e]))
    indptr = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    take = np.concatenate([np.arange(first[u], first[u] + deg[u]) for u in range(V)])
    cd, cw = dest[take], w[take]
    ua, ub, uw = oracle.upper_edges(indptr, cd, cw)
    f = oracle.kruskal_forest(V, ua, ub, uw)
    assert n == f.sum()
    assert set(zip(a.tolist(), b.tolist())) == set(zip(ua[f].tolist(), ub[f].tolist()))
    assert w[ids].astype(np.int64).sum() == uw[f].astype(np.int64).sum()
    return indptr, cd, cw


def _layout_case(layout):
    from masters_final_b200 import workloads as W
    if layout == "high_degree":
        indptr, dest, w = W.knn_graph(20000, k=48, seed=33)
        return indptr[:-1].astype(np.int32), np.diff(indptr).astype(np.int32), dest, w
    indptr, dest, w = W.knn_graph(20000, k=16, seed=31)
    if layout == "parallel":
        return _with_parallel(indptr, dest, w, 32)
    return _layout_permuted(indptr, dest, w, 34)


@pytest.mark.parametrize("layout", ["permuted", "parallel", "high_degree"])
def test_boruvka_csr_layouts(T, layout):
    """Rows out of order with gaps (the row-by-row build), parallel entries
    (the recorded row offsets must still name the first matching entry) and
    rows too long for a warp's row staging (the flat walk): the forest, its
    entry ids and the component labels against the oracle."""
    from masters_final_b200.graph.mst import boruvka_minho_gpu
    from masters_final_b200.graph.connected_components import connected_comps_gpu
    first, deg, dest, w = _layout_case(layout)
    mst, n = boruvka_minho_gpu(dest, w, first, deg)
    indptr, cd, cw = _check_layout(first, deg, dest, w, mst, n)
    labels = connected_comps_gpu(dest, w, first, deg)
    _, ref = oracle.boruvka_seq(indptr, cd, cw)
    assert np.array_equal(labels, ref)


def test_final_clustering_golden(T):
    from masters_final_b200.EAC.eac import sp_sl_lifetime_csr
    for name in ("eac_small", "eac_discard"):
        g = golden(name)
        n = g["x"].shape[0]
        nc, labels = sp_sl_lifetime_csr(g["indptr"], g["indices"], g["diassoc"], n, int(g["P"]))
        assert nc == g["n_fclusts"]
        assert np.array_equal(labels, g["final_labels"])


def test_final_clustering_disconnected(T):
    """Isolated points and separate groups exercise the disconnected-graph
    branch of the lifetime rule (MyML/MyML/EAC/eac.py:238-248)."""
    from masters_final_b200.EAC.eac import sp_sl_lifetime_csr
    rng = np.random.default_rng(3)
    n = 5000
    groups = rng.integers(0, 7, n)
    groups[:50] = -1                      # isolated
    a, b = [], []
    for gidx in range(7):
        m = np.nonzero(groups == gidx)[0]
        for _ in range(6):
            x, y = rng.choice(m, 2 * m.size).reshape(2, -1)
            keep = x != y
            a.append(np.minimum(x, y)[keep])
            b.append(np.maximum(x, y)[keep])
    a, b = np.concatenate(a), np.concatenate(b)
    key = np.unique(a * n + b)
    a, b = key // n, key % n
    w = rng.integers(1, 30, a.size).astype(np.uint8)
    order = np.lexsort((b, a))
    a, b, w = a[order], b[order], w[order]
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(a, minlength=n), out=indptr[1:])
    for P in (29, 40):
        nc, labels = sp_sl_lifetime_csr(indptr, b.astype(np.int32), w, n, P)
        nc2, lab2 = oracle.sp_sl_lifetime(n, a, b, w, P)
        assert nc == nc2
        assert np.array_equal(labels, lab2)


def test_final_clustering_capacity_split_phases(T):
    """More entries than the final clustering's edge array holds at once, with
    one weight owning most of them: the workspace stays below the matrix's
    own size and the forest and the labels do not change."""
    from masters_final_b200 import _lib
    from masters_final_b200.EAC.eac import sp_sl_lifetime_csr
    rng = np.random.default_rng(8)
    n = 12_000
    m = 4_000_000                                   # ~3.7M entries > the edge array (256 n words)
    a = rng.integers(0, n - 1, m)
    b = a + 1 + (rng.random(m) * (n - 1 - a)).astype(np.int64)
    key = np.unique(a * n + b)
    a, b = key // n, key % n
    w = rng.integers(1, 60, a.size).astype(np.uint8)
    w[rng.random(a.size) < 0.7] = 45                # one weight holds ~70% of the entries
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(a, minlength=n), out=indptr[1:])
    L = _lib.load()
    assert L.eacb_final_clustering_workspace_size(n, a.size) < 12 * a.size
    for P in (59, 80):
        nc, labels = sp_sl_lifetime_csr(indptr, b.astype(np.int32), w, n, P)
        nc2, lab2 = oracle.sp_sl_lifetime(n, a, b, w, P)
        assert nc == nc2
        if nc > 1:
            assert np.array_equal(labels, lab2)


def test_final_clustering_overflow_retry(T):
    """A complete graph whose lightest weights hold more entries than the edge
    array: the first phase overflows, is redone as weight pieces, and the
    piece of weight 2 overflows again and is redone as row ranges.  Forest
    and labels must equal the oracle's."""
    from masters_final_b200 import _lib
    from masters_final_b200.EAC.eac import sp_sl_lifetime_csr
    rng = np.random.default_rng(12)
    n = 2400
    a, b = np.triu_indices(n, 1)
    m = a.size                                      # 2,878,800 entries
    group = rng.integers(0, 2, n)                   # two groups joined by heavy entries
    inside = group[a] == group[b]
    w = np.where(inside, rng.integers(3, 60, m), rng.integers(150, 200, m)).astype(np.uint8)
    pick = rng.permutation(np.nonzero(inside)[0])
    w[pick[:10_000]] = 1
    w[pick[10_000:1_210_000]] = 2                   # 1.2M entries (words) > 2^20
    L = _lib.load()
    assert L.eacb_final_clustering_workspace_size(n, m) < 8 * 2 * m
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(a, minlength=n), out=indptr[1:])
    for P in (199, 250):
        nc, labels = sp_sl_lifetime_csr(indptr, b.astype(np.int32), w, n, P)
        nc2, lab2 = oracle.sp_sl_lifetime(n, a.astype(np.int64), b.astype(np.int64), w, P)
        assert nc == nc2
        if nc > 1:
            assert np.array_equal(labels, lab2)
