"""GPU parity of the sparse co-association build (EAC_CSR) against the
reference's outputs and the oracle."""
import hashlib

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


def _build(L, n, max_assocs, kind="linear"):
    from masters_final_b200.EAC.sparse import EAC_CSR
    c = EAC_CSR(n, int(max_assocs), max_assocs_type=kind, condensed=True, sort_mode="surgical")
    c.update_ensemble(L)
    return c


@pytest.mark.parametrize("name", ["eac_small", "eac_discard"])
def test_coassoc_golden(T, name):
    g = golden(name)
    n = g["x"].shape[0]
    c = _build(g["labels_matrix"], n, g["max_assocs"])
    assert c.nnz == g["nnz"]
    assert c.nnz_discarded == g["nnz_discarded"]
    c.make_diassoc()
    assert np.array_equal(c.indptr.cpu().numpy(), g["indptr"])
    assert np.array_equal(c.indices.cpu().numpy(), g["indices"])
    assert np.array_equal(c.data.cpu().numpy(), g["diassoc"])


def test_coassoc_10k_golden(T):
    g = golden("eac_10k")
    n = g["x"].shape[0]
    L = g["labels_matrix"].astype(np.int32)
    c = _build(L, n, g["max_assocs"])
    assert c.nnz == g["nnz"] and c.nnz_discarded == g["nnz_discarded"]
    c.make_diassoc()
    h = hashlib.sha256()
    for a in (c.indptr.cpu().numpy(), c.indices.cpu().numpy(), c.data.cpu().numpy()):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == str(g["coassoc_sha"])


def _random_labels(rng, P, n, kmin, kmax, holes=0.0):
    L = np.empty((P, n), dtype=np.int32)
    for p in range(P):
        k = int(rng.integers(kmin, kmax + 1))
        L[p] = rng.integers(0, k, n)
        if holes:
            L[p][rng.random(n) < holes] = -1
    return L


@pytest.mark.parametrize("seed,n,P,kmin,kmax,factor,kind,holes", [
    (1, 3000, 20, 5, 40, 3, "linear", 0.0),
    (2, 5000, 37, 2, 9, 1, "linear", 0.0),          # tight: discards
    (3, 4000, 12, 30, 300, 2, "constant", 0.05),    # -1 labels, constant caps
    (4, 200_000, 6, 3000, 4000, 3, "linear", 0.0),  # several column chunks per row
    (5, 2500, 255, 10, 20, 3, "linear", 0.0),       # maximum ensemble size
    (6, 36_000, 5, 30, 50, 1, "linear", 0.0),       # capped rows over several chunks
])
def test_coassoc_vs_oracle(T, seed, n, P, kmin, kmax, factor, kind, holes):
    rng = np.random.default_rng(seed)
    L = _random_labels(rng, P, n, kmin, kmax, holes)
    ma = oracle.max_cluster_size(L) * factor
    cap = oracle.indptr_linear(n, ma) if kind == "linear" else oracle.indptr_constant(n, ma)
    ip, ind, cnt, nnz, disc, st = oracle.coassoc_build(L, cap)
    if st == oracle.ERR_FIRST_OVERFLOW:
        from masters_final_b200.EAC.sparse import EAC_CSR
        with pytest.raises(ValueError):
            _build(L, n, ma, kind)
        return
    assert st == 0
    c = _build(L, n, ma, kind)
    assert c.nnz == nnz and c.nnz_discarded == disc
    assert np.array_equal(c.indptr.cpu().numpy(), ip)
    assert np.array_equal(c.indices.cpu().numpy(), ind)
    assert np.array_equal(c.data.cpu().numpy(), cnt)


def _clustered_labels(rng, P, n, groups, split, holes=0.0):
    """Labels with the structure of an EAC ensemble: every partition splits
    each of `groups` point groups into a few clusters of its own."""
    g = rng.integers(0, groups, n)
    L = np.empty((P, n), dtype=np.int32)
    for p in range(P):
        s = int(rng.integers(split[0], split[1] + 1))
        L[p] = g * s + rng.integers(0, s, n)
        if holes:
            L[p][rng.random(n) < holes] = -1
    return L


PATH_CASES = [
    # labels, seed, n, P, (k range | groups, split range), factor, capacity, holes
    ("random", 1, 3000, 20, (5, 40), 3, "linear", 0.0),
    ("random", 2, 5000, 37, (2, 9), 1, "linear", 0.0),          # discards: capped rows
    ("random", 3, 4000, 12, (30, 300), 2, "constant", 0.05),    # -1 labels
    ("random", 5, 2500, 255, (10, 20), 3, "linear", 0.0),       # 255 partitions
    ("clustered", 7, 20000, 50, (40, 3, 6), 3, "linear", 0.0),  # EAC-like structure
    ("clustered", 8, 8000, 100, (12, 2, 5), 1, "linear", 0.02),  # discards and holes
    ("clustered", 9, 550_000, 2, (500, 1, 4), 3, "linear", 0.0),  # neighbourhoods over chunks
]
_PATH_REF = {}


def _path_case(case):
    kind_l, seed, n, P, shape, factor, kind, holes = case
    if case not in _PATH_REF:
        rng = np.random.default_rng(seed)
        if kind_l == "random":
            L = _random_labels(rng, P, n, shape[0], shape[1], holes)
        else:
            L = _clustered_labels(rng, P, n, shape[0], shape[1:], holes)
        ma = oracle.max_cluster_size(L) * factor
        cap = oracle.indptr_linear(n, ma) if kind == "linear" else oracle.indptr_constant(n, ma)
        _PATH_REF.clear()
        _PATH_REF[case] = (L, ma, oracle.coassoc_build(L, cap))
    return _PATH_REF[case]


@pytest.mark.parametrize("ratio", [0, 10 ** 9])
@pytest.mark.parametrize("case", PATH_CASES, ids=[f"{c[0]}{c[1]}" for c in PATH_CASES])
def test_coassoc_paths_vs_oracle(T, case, ratio):
    """The same build with every group forced onto the streaming kernels
    (ratio 0) and onto the pair tiles (ratio 1e9; capped rows still stream)
    equals the oracle."""
    from masters_final_b200 import _lib
    L, ma, (ip, ind, cnt, nnz, disc, st) = _path_case(case)
    assert st == 0
    with _lib.forced("co_dense_ratio", ratio):
        c = _build(L, case[2], ma, case[6])
    assert c.nnz == nnz and c.nnz_discarded == disc
    assert np.array_equal(c.indptr.cpu().numpy(), ip)
    assert np.array_equal(c.indices.cpu().numpy(), ind)
    assert np.array_equal(c.data.cpu().numpy(), cnt)


@pytest.mark.parametrize("ratio", [0, 10 ** 9])
@pytest.mark.parametrize("n,P,k,holes", [(2, 1, 1, 0.0), (7, 3, 2, 0.0), (129, 1, 4, 0.0),
                                         (130, 4, 3, 0.3), (257, 2, 1, 0.0), (300, 5, 40, 0.9)])
def test_coassoc_paths_small_shapes(T, ratio, n, P, k, holes):
    """Shapes at the edges of the pair tiles: fewer rows than one tile,
    one row past a tile, a single partition, one cluster holding every
    point, and mostly unlabelled points; both paths equal the oracle."""
    from masters_final_b200 import _lib
    rng = np.random.default_rng(n * 31 + P)
    L = _random_labels(rng, P, n, k, k, holes)
    ma = max(oracle.max_cluster_size(L), 1) * 3
    cap = oracle.indptr_linear(n, ma)
    ip, ind, cnt, nnz, disc, st = oracle.coassoc_build(L, cap)
    if st != 0:
        pytest.skip("the first partition overflows its capacity")
    with _lib.forced("co_dense_ratio", ratio):
        c = _build(L, n, ma)
    assert c.nnz == nnz and c.nnz_discarded == disc
    assert np.array_equal(c.indptr.cpu().numpy(), ip)
    assert np.array_equal(c.indices.cpu().numpy(), ind)
    assert np.array_equal(c.data.cpu().numpy(), cnt)


@pytest.mark.parametrize("name", ["eac_small", "eac_discard", "eac_10k"])
def test_coassoc_golden_pair_tiles(T, name):
    """The reference-run fixtures with every group on the pair tiles."""
    from masters_final_b200 import _lib
    g = golden(name)
    n = g["x"].shape[0]
    with _lib.forced("co_dense_ratio", 10 ** 9):
        c = _build(g["labels_matrix"].astype(np.int32), n, g["max_assocs"])
    assert c.nnz == g["nnz"] and c.nnz_discarded == g["nnz_discarded"]
    c.make_diassoc()
    if name == "eac_10k":
        h = hashlib.sha256()
        for arr in (c.indptr.cpu().numpy(), c.indices.cpu().numpy(), c.data.cpu().numpy()):
            h.update(np.ascontiguousarray(arr).tobytes())
        assert h.hexdigest() == str(g["coassoc_sha"])
    else:
        assert np.array_equal(c.indptr.cpu().numpy(), g["indptr"])
        assert np.array_equal(c.indices.cpu().numpy(), g["indices"])
        assert np.array_equal(c.data.cpu().numpy(), g["diassoc"])


def test_first_partition_overflow_raises(T):
    from masters_final_b200.EAC.sparse import EAC_CSR
    n = 1000
    L = np.zeros((3, n), dtype=np.int32)          # one cluster holding everything
    L[1] = np.arange(n) % 7
    L[2] = np.arange(n) % 5
    cap_small = 10
    st = oracle.coassoc_build(L, oracle.indptr_constant(n, cap_small))[-1]
    assert st == oracle.ERR_FIRST_OVERFLOW
    with pytest.raises(ValueError):
        _build(L, n, cap_small, "constant")


@pytest.mark.parametrize("kind", ["linear", "constant"])
def test_coassoc_checksum_full_size(T, kind):
    """n = 500,000 points, 20 partitions with k in [350, 710] (the size of the
    BF16 workload, fewer partitions).  Every co-clustered pair is either
    counted in a kept entry or in nnz_discarded (random labels overflow the
    linear capacities, so most rows take the capped path; a constant capacity
    of n keeps everything); rows are strictly increasing and every column
    exceeds its row."""
    rng = np.random.default_rng(9)
    n, P = 500_000, 20
    L = _random_labels(rng, P, n, 350, 710)
    pairs = 0
    for p in range(P):
        s = np.bincount(L[p]).astype(np.int64)
        pairs += int((s * (s - 1) // 2).sum())
    ma = oracle.max_cluster_size(L) * 3 if kind == "linear" else n
    c = _build(L, n, ma, kind)
    if kind == "constant":
        assert c.nnz_discarded == 0
    ip = c.indptr.cpu().numpy()
    ind = c.indices.cpu().numpy()
    dat = c.data.cpu().numpy()
    assert int(dat.astype(np.int64).sum()) + c.nnz_discarded == pairs
    rows = np.repeat(np.arange(n), np.diff(ip))
    assert np.all(ind > rows)
    same = rows[1:] == rows[:-1]
    assert np.all(ind[1:][same] > ind[:-1][same])
    if kind == "linear":
        cap = oracle.indptr_linear(n, ma)
        assert np.all(np.diff(ip) <= np.diff(cap))
