"""K-Means (Lloyd) on the GPU with the reference's exact arithmetic.

Drop-in for MyML/MyML/cluster/KMeans.py:26-201 (``K_Means``).  Same
constructor arguments, the same random initial sample (``random.sample``,
:196), the same stop rule (max_iter label passes, or an inertia change of at
most tol) and the same outputs (``labels_``, ``cluster_centers_``,
``iters_``, ``inertia_``).  Labels equal the reference's for any input.

label_mode: every reference mode ('python', 'numpy', 'numba', 'cuda') runs the
float32 CUDA-core labeler; 'bf16' runs the tcgen05 tensor-core labeler (same
labels).  centroid_mode: 'numba' / 'python' (float32 sums in point order, the
reference's arithmetic) or 'f64' (float64 sums).
"""
import ctypes
import random

import numpy as np

from .. import _lib

_LABEL = {"python": 0, "numpy": 0, "numba": 0, "cuda": 0, "fp32": 0, "bf16": 1, "tc": 1}
_CENTROID = {"python": 0, "numba": 0, "f64": 1}


def kmeans_ensemble(X, ks, inits, max_iter=3, tol=1e-4, label_mode="cuda",
                    centroid_mode="numba", converge=True, stream=None):
    """Run len(ks) independent fits on the same data in one batched pass.
    X: (n, d) float32 (numpy or CUDA tensor); ks: list of k; inits: list of
    initial sample index lists.  Returns device tensors
    (labels P x n, centroids P x kmax x d, dists P x n, iters P, inertia P)."""
    t = _lib.torch()
    Xd = _lib.to_device(X, t.float32)
    n, d = int(Xd.shape[0]), int(Xd.shape[1])
    P = len(ks)
    kmax = int(max(ks))
    dev = Xd.device
    k_d = t.tensor(np.asarray(ks, dtype=np.int32), device=dev)
    init = np.zeros((P, kmax), dtype=np.int32)
    for p, idx in enumerate(inits):
        init[p, :len(idx)] = idx
    init_d = t.from_numpy(init).to(dev)
    labels = t.empty((P, n), dtype=t.int32, device=dev)
    cent = t.zeros((P, kmax, d), dtype=t.float32, device=dev)
    dists = t.empty((P, n), dtype=t.float32, device=dev)
    iters = t.empty(P, dtype=t.int32, device=dev)
    inertia = t.empty(P, dtype=t.float32, device=dev)
    L = _lib.load()
    ws = _lib.workspace(L.eacb_kmeans_workspace_size(n, d, P, kmax))
    mode = _LABEL[label_mode]
    cmode = _CENTROID[centroid_mode]
    tol_f = float(np.float32(tol)) if converge else -1.0
    _lib.check(L.eacb_kmeans_ensemble(_lib.ptr(Xd), n, d, P, _lib.ptr(k_d), kmax, _lib.ptr(init_d),
                                      int(max_iter), tol_f, mode, cmode, _lib.ptr(labels),
                                      _lib.ptr(cent), _lib.ptr(dists), _lib.ptr(iters),
                                      _lib.ptr(inertia), _lib.ptr(ws), ws.numel(),
                                      _lib.stream_handle(stream)), "kmeans")
    return labels, cent, dists, iters, inertia


def kmeans_label(X, centroids, label_mode="cuda", stream=None):
    """One label step: (labels, float32 distances) as device tensors."""
    t = _lib.torch()
    Xd = _lib.to_device(X, t.float32)
    Cd = _lib.to_device(centroids, t.float32)
    n, d = int(Xd.shape[0]), int(Xd.shape[1])
    k = int(Cd.shape[0])
    labels = t.empty(n, dtype=t.int32, device=Xd.device)
    dists = t.empty(n, dtype=t.float32, device=Xd.device)
    L = _lib.load()
    ws = _lib.workspace(L.eacb_kmeans_label_workspace_size(n, d, k))
    _lib.check(L.eacb_kmeans_label(_lib.ptr(Xd), n, d, _lib.ptr(Cd), k, _LABEL[label_mode],
                                   _lib.ptr(labels), _lib.ptr(dists), _lib.ptr(ws), ws.numel(),
                                   _lib.stream_handle(stream)), "kmeans label")
    _lib.check(L.eacb_workspace_status(_lib.ptr(ws), _lib.stream_handle(stream)), "kmeans label")
    return labels, dists


def kmeans_centroids(X, labels, dists, k, centroid_mode="numba", stream=None):
    """One centroid update (MyML/MyML/cluster/KMeans.py:709-754): a (k, d)
    float32 device tensor; empty clusters take the points the reference's
    quickselect picks from ``dists``."""
    t = _lib.torch()
    Xd = _lib.to_device(X, t.float32)
    Ld = _lib.to_device(labels, t.int32)
    Dd = _lib.to_device(dists, t.float32)
    n, d = int(Xd.shape[0]), int(Xd.shape[1])
    C = t.empty((int(k), d), dtype=t.float32, device=Xd.device)
    L = _lib.load()
    ws = _lib.workspace(L.eacb_kmeans_centroids_workspace_size(n, d, int(k)))
    _lib.check(L.eacb_kmeans_centroids(_lib.ptr(Xd), n, d, _lib.ptr(Ld), _lib.ptr(Dd), int(k),
                                       _CENTROID[centroid_mode], _lib.ptr(C), _lib.ptr(ws),
                                       ws.numel(), _lib.stream_handle(stream)), "kmeans centroids")
    return C


class K_Means:
    """MyML/MyML/cluster/KMeans.py:26 (same arguments and attributes)."""

    def __init__(self, n_clusters=8, tol=1e-4, max_iter=300, init='random', **kwargs):
        self.n_clusters = n_clusters
        self._label_mode = kwargs.get("label_mode", "cuda")
        self._centroid_mode = kwargs.get("centroid_mode", "numba")
        if self._label_mode not in _LABEL:
            raise ValueError("label_mode should be one of {}".format(list(_LABEL)))
        if self._centroid_mode not in _CENTROID:
            raise ValueError("centroid_mode should be one of {}".format(list(_CENTROID)))
        if isinstance(init, str) and init == 'random':
            self.centroid_init_mode = 'random'
        elif isinstance(init, np.ndarray):
            if init.shape[0] != n_clusters:
                raise Exception("Number of clusters indicated different from number of "
                                "centroids supplied.")
            self.centroid_init_mode = init.copy()
        else:
            raise ValueError("Centroid init may be 'random' or an ndarray containing the "
                             "centroids to use.")
        self.tol = tol
        self.max_iter = max_iter
        self._converge = kwargs.get("converge", True)
        self.inertia_ = np.inf
        self.iters_ = 0
        self.stream = kwargs.get("stream", None)

    def _init_centroids_idx(self, N):
        """Initial sample (MyML/MyML/cluster/KMeans.py:191-201)."""
        return random.sample(range(N), self.n_clusters)

    def fit(self, data):
        data = np.asarray(data) if not hasattr(data, "data_ptr") else data
        if _lib.np_dtype_of(data) != np.float32:
            raise Warning("DATA DUPLICATION: data converted to float32.TODO: accept other formats")
        N, D = int(data.shape[0]), int(data.shape[1])
        self.N, self.D = N, D
        if isinstance(self.centroid_init_mode, str):
            init = self._init_centroids_idx(N)
            labels, cent, dists, iters, inertia = kmeans_ensemble(
                data, [self.n_clusters], [init], self.max_iter, self.tol, self._label_mode,
                self._centroid_mode, self._converge, self.stream)
        else:
            raise NotImplementedError("explicit initial centroids: pass them as sample indices "
                                      "through kmeans_ensemble")
        self.labels_ = labels[0].cpu().numpy()
        self.cluster_centers_ = cent[0, :self.n_clusters].cpu().numpy()
        self.iters_ = int(iters[0].item())
        self.inertia_ = np.float32(inertia[0].item())
        self._dists = dists[0].cpu().numpy()
        return self
