"""Evidence accumulation clustering: final clustering (and the EAC driver).

Drop-in for MyML/MyML/EAC/eac.py.  ``sp_sl_lifetime`` (:199-267) takes the
condensed dissimilarity CSR and returns ``(n_comps, labels)`` with the
reference's conventions; its minimum spanning forest, lifetime rule and
component labelling run in ``eacb_final_clustering`` (libeacb200).
"""
import ctypes

import numpy as np

from .. import _lib


def sp_sl_lifetime_csr(indptr, indices, diassoc, n, max_dist, n_clusters=0,
                       returnDevAry=False, stream=None):
    """Final clustering of an upper-triangle CSR given as arrays (numpy or
    CUDA tensors): int64 indptr (n+1), int32 indices, uint8 dissimilarities.
    Returns (n_fclusts, labels); labels is empty when one cluster results,
    like the reference."""
    t = _lib.torch()
    ip = _lib.to_device(indptr, t.int64)
    ind = _lib.to_device(indices, t.int32)
    dat = _lib.to_device(diassoc, t.uint8)
    nnz = ind.numel()
    L = _lib.load()
    ws = _lib.workspace(L.eacb_final_clustering_workspace_size(n, nnz))
    labels = t.empty(n, dtype=t.int32, device=ip.device)
    nf = ctypes.c_int64(0)
    valid = ctypes.c_int32(0)
    st = L.eacb_final_clustering(_lib.ptr(ip), _lib.ptr(ind), _lib.ptr(dat), n, nnz,
                                 int(max_dist), int(n_clusters), _lib.ptr(labels),
                                 ctypes.byref(nf), ctypes.byref(valid), _lib.ptr(ws),
                                 ws.numel(), _lib.stream_handle(stream))
    if st == _lib.ERR_VALUE:
        raise ValueError("lifetime rule undefined: fewer than two MST edges or no two "
                         "MST edges of equal weight (the reference raises here too)")
    _lib.check(st, "sp_sl_lifetime")
    if not valid.value:
        lab = t.empty(0, dtype=t.int32, device=ip.device)
    else:
        lab = labels
    if returnDevAry:
        return int(nf.value), lab
    return int(nf.value), lab.cpu().numpy()


def sp_sl_lifetime(mat, max_dist=None, n_clusters=0):
    """MyML/MyML/EAC/eac.py:199-267 on a scipy CSR matrix holding the
    condensed (upper-triangle) uint8 dissimilarities."""
    if max_dist is None:
        max_dist = int(mat.data.max())        # the reference then adds 1
    data = np.asarray(mat.data)
    if data.dtype != np.uint8:
        raise TypeError("the co-association dissimilarities must be uint8")
    return sp_sl_lifetime_csr(np.asarray(mat.indptr, dtype=np.int64),
                              np.asarray(mat.indices, dtype=np.int32), data,
                              mat.shape[0], max_dist, n_clusters)


def lifetime_n_clusters(weights):
    """MyML/MyML/EAC/eac.py:366-391: number of clusters by the maximum
    lifetime of sorted MST weights (host utility on a small array; the
    device pipeline evaluates the same rule on the weight histogram)."""
    weights = np.asarray(weights)
    lifetimes = weights[1:] - weights[:-1]
    m_index = np.argmax(lifetimes)
    th = lifetimes[m_index]
    indices = np.where(weights > weights[m_index])[0]
    cont = 1 if indices.size == 0 else indices.size + 1
    close = np.where(np.isclose(lifetimes, 0))
    minimum = np.min(lifetimes[close])
    if th < 2 * minimum:
        cont = 1
    return cont, th
