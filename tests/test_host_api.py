"""Host-side logic of the drop-in API that runs without a GPU: argument
checks with the reference's error types, the host draws of the ensemble,
ensemble format conversion and the lifetime utility."""
import random

import numpy as np
import pytest

import oracle
from tests.conftest import golden


@pytest.mark.parametrize("kwargs, exc", [
    (dict(max_assocs=0), ValueError),
    (dict(max_assocs=2.5), TypeError),
    (dict(max_assocs=10, condensed="yes"), TypeError),
    (dict(max_assocs=10, dtype=str), TypeError),
    (dict(max_assocs=10, sort_mode="quick"), ValueError),
    (dict(max_assocs=10, max_assocs_type="square"), ValueError),
    (dict(max_assocs=10, max_assocs_type="linear", condensed=False), ValueError),
])
def test_eac_csr_option_errors(kwargs, exc):
    """MyML/MyML/EAC/sparse.py:109-138: the same exception types, raised
    before any device work."""
    from masters_final_b200.EAC.sparse import EAC_CSR
    with pytest.raises(exc):
        EAC_CSR(100, **kwargs)


def test_eac_csr_sample_count_errors():
    from masters_final_b200.EAC.sparse import EAC_CSR
    with pytest.raises(ValueError):
        EAC_CSR(0, max_assocs=10)
    with pytest.raises(TypeError):
        EAC_CSR(100.0, max_assocs=10)


def test_draws_follow_the_reference_order():
    """k per partition (np.random.randint, kmax exclusive) then the initial
    samples (random.sample), partition after partition, as the oracle's
    restatement of generateEnsemble + K_Means draws them."""
    from masters_final_b200.utils.partition import draw_ensemble_params
    from masters_final_b200.EAC.batched import draw_instance_params
    for n, kr, P, seed in [(500, [5, 12], 7, 3), (2000, [20, 20], 4, 11), (50, 6, 3, 0)]:
        np.random.seed(seed)
        random.seed(seed)
        ks, inits = draw_ensemble_params(n, kr, P)
        np.random.seed(seed)
        random.seed(seed)
        ref = oracle.draw_ensemble_params(n, kr if isinstance(kr, list) else kr, P)
        assert ks == [k for k, _ in ref]
        assert inits == [list(s) for _, s in ref]
        if isinstance(kr, list):
            ks2, inits2 = draw_instance_params(n, kr, P, seed)
            assert (ks2, inits2) == (ks, inits)


def test_label_matrix_from_ensemble():
    """A list-of-clusters partition (the reference's ensemble format) gives
    each member its cluster's position; points in no cluster get -1."""
    from masters_final_b200.EAC.sparse import label_matrix_from_ensemble
    ens = [[np.array([0, 3]), np.array([1, 2, 4])],
           [np.array([4]), np.array([0, 1]), np.array([2, 3])],
           [np.array([0, 1, 2])]]
    L = label_matrix_from_ensemble(ens, 5)
    assert L.dtype == np.int32 and L.shape == (3, 5)
    assert L.tolist() == [[0, 1, 1, 0, 1], [1, 1, 2, 2, 0], [0, 0, 0, -1, -1]]


def test_lifetime_host_utility_matches_reference():
    """EAC.eac.lifetime_n_clusters on the reference's own outputs."""
    from masters_final_b200.EAC.eac import lifetime_n_clusters
    g = golden("lifetime")
    for t in range(6):
        cont, th = lifetime_n_clusters(g["w%d" % t])
        assert cont == g["cont%d" % t] and th == g["th%d" % t]


def test_dense_path_not_built():
    """The dense co-association path is outside the GPU build and says so."""
    from masters_final_b200.EAC.eac import EAC
    e = EAC(10, sparse=False)
    with pytest.raises(NotImplementedError):
        e.buildMatrix(np.zeros((2, 10), dtype=np.int32))


def test_to_host_empty_result():
    """An empty device result (the final clustering when no labels are
    produced) comes back as an empty array of the same dtype without
    touching the device or the pinned allocator."""
    import torch
    from masters_final_b200 import _lib
    out = _lib.to_host(torch.empty(0, dtype=torch.int32))
    assert isinstance(out, np.ndarray) and out.dtype == np.int32 and out.shape == (0,)
