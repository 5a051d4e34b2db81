"""Failure paths: inputs the device-side checks must refuse, and the bounded
round loop.

The reference has no such checks: a corrupt graph sends its Boruvka loop
(MyML/MyML/graph/mst.py:487-492) around forever or reads out of bounds.
Here every fault is made on the host (a corrupt CSR, a dropped edge
direction, a label past the cluster count, a lowered round cap), each
kernel's own bounds check turns it into an error word, and the Python
wrapper raises EACBError carrying the documented status.  None of these
inputs makes a kernel read or write out of bounds.
"""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

BAD_INPUT, NOT_CONVERGED = -8, -6


@pytest.fixture(scope="module")
def T():
    import torch
    assert torch.cuda.is_available()
    return torch


def _graph(n=2000, k=6, seed=31):
    from masters_final_b200 import workloads as W
    indptr, dest, w = W.knn_graph(n, k=k, seed=seed)
    return indptr, dest.copy(), w.copy()


def _raises(status, fn, *args):
    from masters_final_b200._lib import EACBError
    with pytest.raises(EACBError) as ei:
        fn(*args)
    assert ei.value.status == status, str(ei.value)


@pytest.mark.parametrize("bad", [-2, 2000, 1 << 30])
def test_dest_out_of_range(T, bad):
    from masters_final_b200.graph.mst import boruvka_minho_gpu
    from masters_final_b200.graph.connected_components import connected_comps_gpu
    indptr, dest, w = _graph()
    dest[123] = bad
    first, deg = indptr[:-1].astype(np.int32), np.diff(indptr).astype(np.int32)
    _raises(BAD_INPUT, boruvka_minho_gpu, dest, w, first, deg)
    _raises(BAD_INPUT, connected_comps_gpu, dest, w, first, deg)


def test_row_extent_out_of_range(T):
    from masters_final_b200.graph.mst import boruvka_minho_gpu
    indptr, dest, w = _graph()
    first, deg = indptr[:-1].astype(np.int32), np.diff(indptr).astype(np.int32)
    deg[-1] += 5                                   # last row runs past the entries
    _raises(BAD_INPUT, boruvka_minho_gpu, dest, w, first, deg)


def test_asymmetric_graph(T):
    """A forest edge stored only in the row of its larger endpoint: the edge
    ids are defined in the row of the smaller one, which lacks it."""
    from masters_final_b200 import workloads as W
    from masters_final_b200.graph.mst import boruvka_minho_gpu
    a = np.array([0, 1, 2], dtype=np.int64)
    b = np.array([1, 2, 3], dtype=np.int64)
    indptr, dest, w = W.csr_from_undirected(4, a, b, np.array([3, 1, 2], dtype=np.uint8))
    row1 = slice(indptr[1], indptr[2])
    keep = np.ones(dest.size, dtype=bool)
    keep[row1.start + int(np.flatnonzero(dest[row1] == 2)[0])] = False   # drop 1 -> 2
    rows = np.repeat(np.arange(4), np.diff(indptr))[keep]
    dest, w = dest[keep], w[keep]
    indptr = np.zeros(5, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=4), out=indptr[1:])
    _raises(BAD_INPUT, boruvka_minho_gpu, dest, w, indptr[:-1].astype(np.int32),
            np.diff(indptr).astype(np.int32))


def test_label_past_cluster_count(T):
    """Co-association member lists of a label matrix holding a label >= K."""
    from masters_final_b200 import _lib
    L = _lib.load()
    n, P, K = 5000, 4, 20
    rng = np.random.default_rng(5)
    lab = rng.integers(0, K, size=(P, n)).astype(np.int32)
    lab[2, 777] = K
    d = T.from_numpy(lab).cuda()
    ws = _lib.workspace(L.eacb_coassoc_workspace_size(n, P, K))
    mc = ctypes.c_int64(0)
    st = L.eacb_coassoc_prepare(_lib.ptr(d), n, P, K, ctypes.byref(mc), _lib.ptr(ws), ws.numel(),
                                _lib.stream_handle())
    assert st == BAD_INPUT, _lib.status_string(st)
    # the same matrix without the bad label goes through
    lab[2, 777] = 3
    d = T.from_numpy(lab).cuda()
    st = L.eacb_coassoc_prepare(_lib.ptr(d), n, P, K, ctypes.byref(mc), _lib.ptr(ws), ws.numel(),
                                _lib.stream_handle())
    assert st == 0
    assert mc.value == oracle.max_cluster_size(lab)


def test_round_cap_reports_not_converged(T):
    """A valid graph that needs more Boruvka rounds than allowed: the round
    kernel stops at the cap and the call reports EACB_ERR_NOT_CONVERGED
    instead of looping; with the cap lifted the same graph succeeds."""
    from masters_final_b200 import _lib
    from masters_final_b200.graph.mst import boruvka_minho_gpu
    from masters_final_b200.graph.connected_components import connected_comps_gpu
    indptr, dest, w = _graph(20000, 8, 41)
    first, deg = indptr[:-1].astype(np.int32), np.diff(indptr).astype(np.int32)
    L = _lib.load()
    L.eacb_debug_set_round_cap(1)
    try:
        _raises(NOT_CONVERGED, boruvka_minho_gpu, dest, w, first, deg)
        _raises(NOT_CONVERGED, connected_comps_gpu, dest, w, first, deg)
    finally:
        L.eacb_debug_set_round_cap(0)
    # with the cap lifted, the next calls (fresh workspaces) are exact again
    _, ref = oracle.boruvka_seq(indptr, dest, w)
    mst, n = boruvka_minho_gpu(dest, w, first, deg)
    assert n == 20000 - np.unique(ref).size
    assert np.array_equal(connected_comps_gpu(dest, w, first, deg), ref)
