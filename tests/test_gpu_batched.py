"""GPU parity of the batched EAC (many instances in one call) against the
reference's golden end-to-end results and the oracle pipeline."""
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


def _golden_instances():
    from masters_final_b200.EAC.batched import draw_instance_params
    gs = [golden(n) for n in ("eac_small", "eac_discard", "eac_10k")]
    params = [draw_instance_params(g["x"].shape[0], [int(g["kmin"]), int(g["kmax"])], int(g["P"]),
                                   int(g["seed"])) for g in gs]
    return gs, params


@pytest.mark.parametrize("mode", ["cuda", "bf16"])
def test_batched_goldens(T, mode):
    """Three reference EAC runs (one with discarded associations) in one
    batched call: kept/discarded counts, cluster count and labels exact."""
    from masters_final_b200.EAC.batched import eac_batch
    gs, params = _golden_instances()
    # eac_discard uses factor 1, the others 3: one call per factor
    for factor in (1, 3):
        sel = [i for i, g in enumerate(gs) if int(g["factor"]) == factor]
        res = eac_batch([gs[i]["x"] for i in sel], params=[params[i] for i in sel],
                        label_mode=mode, max_assocs_factor=factor, n_workers=4)
        for i, r in zip(sel, res):
            g = gs[i]
            assert r.status == 0
            assert r.nnz == g["nnz"]
            assert r.nnz_discarded == g["nnz_discarded"]
            assert r.n_fclusts == g["n_fclusts"]
            assert np.array_equal(r.labels, g["final_labels"])


def _oracle_eac(x, params, factor=3):
    """The reference pipeline restated on the CPU (oracle)."""
    ks, inits = params
    L = oracle.ensemble_labels(x, list(zip(ks, inits)))
    n = x.shape[0]
    cap = oracle.indptr_linear(n, oracle.max_cluster_size(L) * factor)
    indptr, indices, counts, nnz, disc, st = oracle.coassoc_build(L, cap)
    assert st == 0
    w = (int(counts.max()) + 1 - counts.astype(np.int64)).astype(np.uint8)
    a = np.repeat(np.arange(n), np.diff(indptr)).astype(np.int64)
    nc, labels = oracle.sp_sl_lifetime(n, a, indices.astype(np.int64), w, len(ks))
    if nc <= 1:
        labels = np.zeros(n, dtype=np.int32)
    return nc, labels, nnz, disc


def _random_instances(m, seed):
    from masters_final_b200 import workloads as W
    from masters_final_b200.EAC.batched import draw_instance_params
    rng = np.random.default_rng(seed)
    xs, params = [], []
    for i in range(m):
        n = int(rng.integers(300, 2500))
        d = int(rng.choice([2, 4, 8, 16, 32]))
        comps = int(rng.integers(3, 12))
        x = W.gaussian_mixture(n, d, comps, seed=1000 * seed + i, anisotropic=False,
                               center_range=10.0, sigma=float(rng.uniform(0.5, 2.0)))
        kmin = int(np.ceil(np.sqrt(n) / 2))
        kmax = int(np.ceil(np.sqrt(n)))
        xs.append(x)
        params.append(draw_instance_params(n, [kmin, kmax], 20, 77 + i))
    return xs, params


def test_batched_vs_oracle(T):
    """Ten instances of uneven n and d (the batched workload's shape at small
    sizes): every final partition equals the oracle's."""
    from masters_final_b200.EAC.batched import eac_batch
    xs, params = _random_instances(10, seed=5)
    res = eac_batch(xs, params=params, label_mode="bf16", n_workers=6)
    for x, p, r in zip(xs, params, res):
        nc, labels, nnz, disc = _oracle_eac(x, p)
        assert r.status == 0
        assert (r.nnz, r.nnz_discarded) == (nnz, disc)
        assert r.n_fclusts == nc
        assert np.array_equal(r.labels, labels)


def test_batched_small_arena_serialises(T):
    """An arena that holds only the largest instance's block makes workers
    wait for one another; the results do not change."""
    from masters_final_b200 import _lib
    from masters_final_b200.EAC.batched import eac_batch
    xs, params = _random_instances(8, seed=9)
    ref = eac_batch(xs, params=params, n_workers=8)
    L = _lib.load()
    need = 0
    for x, r in zip(xs, ref):
        n = x.shape[0]
        b = (-(-r.nnz * 4 // 256) * 256 + -(-r.nnz // 256) * 256
             + L.eacb_final_clustering_workspace_size(n, r.nnz))
        need = max(need, b)
    res = eac_batch(xs, params=params, n_workers=8, arena_bytes=need + 256)
    for a, b in zip(ref, res):
        assert b.status == 0
        assert np.array_equal(a.labels, b.labels)
        assert a.n_fclusts == b.n_fclusts


def test_batched_arena_too_small_reports(T):
    """An instance whose block cannot fit gets EACB_ERR_WORKSPACE; the call
    raises with every instance's own status."""
    from masters_final_b200 import _lib
    from masters_final_b200.EAC.batched import eac_batch
    xs, params = _random_instances(3, seed=11)
    with pytest.raises(_lib.EACBError) as ei:
        eac_batch(xs, params=params, n_workers=2, arena_bytes=4096)
    st = [r.status for r in ei.value.results]
    assert all(s == -2 for s in st)
