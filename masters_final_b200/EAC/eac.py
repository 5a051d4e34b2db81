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
    return int(nf.value), _lib.to_host(lab)


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


def lifetime_cut_gpu(mst_weights, n_samples, max_dist, n_clusters=0, stream=None):
    """The lifetime rule and cut decision of sp_sl_lifetime on the device
    (MyML/MyML/EAC/eac.py:220-265, 366-391): (number of clusters, largest
    forest weight kept) for the uint8 weights of a minimum spanning forest of
    n_samples points.  Raises ValueError where the reference does."""
    t = _lib.torch()
    W = _lib.to_device(mst_weights, t.uint8)
    L = _lib.load()
    ws = _lib.workspace(L.eacb_lifetime_cut_workspace_size())
    nc, th = ctypes.c_int64(0), ctypes.c_int32(0)
    st = L.eacb_lifetime_cut(_lib.ptr(W), int(W.numel()), int(n_samples), int(max_dist),
                             int(n_clusters), ctypes.byref(nc), ctypes.byref(th), _lib.ptr(ws),
                             ws.numel(), _lib.stream_handle(stream))
    if st == _lib.ERR_VALUE:
        raise ValueError("lifetime rule undefined: fewer than two MST edges or no two MST "
                         "edges of equal weight (the reference raises here too)")
    _lib.check(st, "lifetime cut")
    return int(nc.value), int(th.value)


def relabel_canonical(labels, stream=None):
    """Numbers groups by their smallest member (scipy connected_components'
    numbering); returns (device int32 labels, number of groups)."""
    t = _lib.torch()
    Ld = _lib.to_device(labels, t.int32)
    n = int(Ld.numel())
    out = t.empty_like(Ld)
    L = _lib.load()
    ws = _lib.workspace(L.eacb_relabel_canonical_workspace_size(n))
    ng = ctypes.c_int64(0)
    _lib.check(L.eacb_relabel_canonical(_lib.ptr(Ld), n, _lib.ptr(out), ctypes.byref(ng),
                                        _lib.ptr(ws), ws.numel(), _lib.stream_handle(stream)),
               "relabel")
    return out, int(ng.value)


class EAC:
    """Evidence accumulation clustering (MyML/MyML/EAC/eac.py:40-179).

    Same keyword arguments; the sparse path (``sparse=True``) is the one built
    on the GPU.  ``buildMatrix`` accepts the reference's list-of-clusters
    ensemble or a (P x n) label matrix (numpy or CUDA tensor)."""

    def __init__(self, n_samples, **kwargs):
        self.n_samples = n_samples
        self.n_partitions = kwargs.get("n_partitions", 100)
        self.iters = kwargs.get("iters", 3)
        self.n_clusters = kwargs.get("n_clusters", "sqrt")
        self.condensed = kwargs.get("condensed", True)
        self.kNN = kwargs.get("kNN", False)
        self.assoc_dtype = kwargs.get("assoc_dtype", np.uint8)
        self.sparse = kwargs.get("sparse", False)
        self.sp_sort = kwargs.get("sparse_sort_mode", "surgical")
        self.sp_max_assocs = kwargs.get("sparse_max_assocs", None)
        self.sp_max_assocs_factor = kwargs.get("sparse_max_assocs_factor", 3)
        self.sp_max_assocs_mode = kwargs.get("sparse_max_assocs_mode", "linear")
        self.sp_keep_degree = kwargs.get("sparse_keep_degree", False)
        self.full = not self.sparse and not self.kNN
        self.coassoc_store = kwargs.get("coassoc_store", False)
        self.linkage = kwargs.get("linkage", "SL")
        self.disk_mst = kwargs.get("sl_disk", False)
        self.stream = kwargs.get("stream", None)

    def buildMatrix(self, ensemble):
        from .sparse import EAC_CSR, CoassocBuilder, label_matrix_from_ensemble
        if not self.sparse:
            raise NotImplementedError("the dense co-association path is not part of the GPU "
                                      "build; use sparse=True")
        if self.disk_mst or self.coassoc_store:
            raise NotImplementedError("disk-backed storage is not part of the GPU build")
        t = _lib.torch()
        labels = ensemble
        if not isinstance(ensemble, (np.ndarray, t.Tensor)):
            labels = label_matrix_from_ensemble(ensemble, self.n_samples)
        builder = CoassocBuilder(labels, self.n_samples, stream=self.stream)
        if self.sp_max_assocs is None:
            self.sp_max_assocs = builder.max_cluster * self.sp_max_assocs_factor
        coassoc = EAC_CSR(self.n_samples, max_assocs=int(self.sp_max_assocs),
                          condensed=self.condensed, max_assocs_type=self.sp_max_assocs_mode,
                          sort_mode=self.sp_sort, dtype=self.assoc_dtype, stream=self.stream)
        coassoc.update_ensemble(None, builder=builder)
        coassoc._condense(keep_degree=self.sp_keep_degree)
        coassoc.make_diassoc()
        self.coassoc = coassoc

    def finalClustering(self, n_clusters=0):
        if not self.sparse:
            raise NotImplementedError("the dense co-association path is not part of the GPU build")
        c = self.coassoc
        n_fclusts, labels = sp_sl_lifetime_csr(c.indptr, c.indices, c.data, self.n_samples,
                                               self.n_partitions, n_clusters=n_clusters,
                                               stream=self.stream)
        self.n_fclusts = n_fclusts
        self.labels = labels
        return labels


def eac_pipeline(X, n_partitions, n_clusters, iters=3, label_mode="cuda",
                 centroid_mode="numba", factor=3, stream=None):
    """Ensemble (batched K-Means) -> sparse co-association -> Boruvka MST ->
    lifetime cut, all on the device.  Returns (n_fclusts, labels, eac)."""
    from ..utils.partition import generate_ensemble_labels
    n = int(X.shape[0])
    L, _ = generate_ensemble_labels(X, n_clusters, n_partitions, iters, label_mode=label_mode,
                                    centroid_mode=centroid_mode, stream=stream)
    eac = EAC(n, sparse=True, condensed=True, n_partitions=n_partitions,
              sparse_max_assocs_factor=factor, stream=stream)
    eac.buildMatrix(L)
    labels = eac.finalClustering()
    return eac.n_fclusts, labels, eac
