"""Sparse (condensed CSR) co-association matrix on the GPU.

Drop-in for MyML/MyML/EAC/sparse.py:12-304 (``EAC_CSR``).  The build runs in
libeacb200 (``eacb_coassoc_prepare/count/fill``) and reproduces the
reference's result exactly -- counts, row order, per-row capacity and the
discarded-association count -- without its per-pair insertion sort.

Accepted ensembles: the reference's list of partitions, each a list of
member-index arrays (convertClusterStringToIndex format), or a label matrix
(P x n, cluster id per point, -1 = none) as a numpy array or CUDA tensor; the
GPU ensemble generator produces the latter directly.
"""
import ctypes

import numpy as np

from .. import _lib


def _compute_max_assocs_from_ensemble(ensemble):
    """MyML/MyML/EAC/sparse.py:1065-1066 for a list-of-clusters ensemble."""
    return max([max(map(np.size, p)) for p in ensemble])


def label_matrix_from_ensemble(ensemble, n_samples):
    """(P x n int32) cluster-index matrix of a list-of-clusters ensemble;
    cluster c of partition p gets id c (its position in the list)."""
    P = len(ensemble)
    L = np.full((P, n_samples), -1, dtype=np.int32)
    for p, part in enumerate(ensemble):
        for c, members in enumerate(part):
            L[p, np.asarray(members, dtype=np.int64)] = c
    return L


class CoassocBuilder:
    """Device-side state shared by the three build calls."""

    def __init__(self, labels, n_samples, n_clusters_max=None, stream=None):
        t = _lib.torch()
        self.L = _lib.to_device(labels, t.int32)
        if self.L.dim() != 2 or self.L.shape[1] != n_samples:
            raise ValueError("label matrix must be P x n_samples")
        self.P = int(self.L.shape[0])
        self.n = int(n_samples)
        if n_clusters_max is None:
            n_clusters_max = int(self.L.max().item()) + 1
        self.K = max(int(n_clusters_max), 1)
        self.stream = stream
        lib = _lib.load()
        self.ws = _lib.workspace(lib.eacb_coassoc_workspace_size(self.n, self.P, self.K))
        mc = ctypes.c_int64(0)
        _lib.check(lib.eacb_coassoc_prepare(_lib.ptr(self.L), self.n, self.P, self.K,
                                            ctypes.byref(mc), _lib.ptr(self.ws), self.ws.numel(),
                                            _lib.stream_handle(stream)), "coassoc prepare")
        self.max_cluster = int(mc.value)

    def build(self, cap_indptr):
        t = _lib.torch()
        lib = _lib.load()
        dev = self.L.device
        indptr = t.empty(self.n + 1, dtype=t.int64, device=dev)
        nnz = ctypes.c_int64(0)
        st = lib.eacb_coassoc_count(_lib.ptr(self.L), self.n, self.P, self.K, _lib.ptr(cap_indptr),
                                    _lib.ptr(indptr), ctypes.byref(nnz), _lib.ptr(self.ws),
                                    self.ws.numel(), _lib.stream_handle(self.stream))
        if st == _lib.ERR_FIRST_OVERFLOW:
            raise ValueError("a row of the first partition exceeds its capacity; the reference "
                             "(MyML/MyML/EAC/sparse.py:446-465) would write past the row")
        _lib.check(st, "coassoc count")
        nnz = int(nnz.value)
        indices = t.empty(max(nnz, 1), dtype=t.int32, device=dev)
        data = t.empty(max(nnz, 1), dtype=t.uint8, device=dev)
        disc = ctypes.c_int64(0)
        mx = ctypes.c_int32(0)
        _lib.check(lib.eacb_coassoc_fill(_lib.ptr(self.L), self.n, self.P, self.K,
                                         _lib.ptr(cap_indptr), _lib.ptr(indptr), _lib.ptr(indices),
                                         _lib.ptr(data), 0, ctypes.byref(disc), ctypes.byref(mx),
                                         _lib.ptr(self.ws), self.ws.numel(),
                                         _lib.stream_handle(self.stream)), "coassoc fill")
        return indptr, indices[:nnz], data[:nnz], nnz, int(disc.value), int(mx.value)


def capacity_indptr(n_samples, max_assocs, max_assocs_type="linear", n_s=0.05, n_e=1.0,
                    val_s=1.0, val_e=0.05, stream=None):
    """Device int64 capacity layout (indptr_linear / indptr_constant)."""
    t = _lib.torch()
    lib = _lib.load()
    cap = t.empty(n_samples + 1, dtype=t.int64, device=_lib.device())
    if max_assocs_type == "constant":
        _lib.check(lib.eacb_capacity_constant(n_samples, int(max_assocs), _lib.ptr(cap),
                                              _lib.stream_handle(stream)), "capacity")
    else:
        ws = _lib.workspace(lib.eacb_capacity_workspace_size(n_samples))
        _lib.check(lib.eacb_capacity_linear(n_samples, int(max_assocs), float(n_s), float(n_e),
                                            float(val_s), float(val_e), _lib.ptr(cap),
                                            _lib.ptr(ws), ws.numel(), _lib.stream_handle(stream)),
                   "capacity")
    return cap


class EAC_CSR:
    """Condensed sparse co-association matrix (MyML/MyML/EAC/sparse.py:12).

    Arrays live on the GPU: ``indptr`` (int64, n+1), ``indices`` (int32),
    ``data`` (uint8).  ``csr`` (a scipy matrix on the host) is built on
    first access."""

    def __init__(self, n_samples, max_assocs, max_assocs_type="constant", dtype=np.uint8,
                 condensed=False, sort_mode="numpy", **kwargs):
        self.n_samples = n_samples
        self.max_assocs = max_assocs
        self.max_assocs_type = max_assocs_type
        self.dtype = dtype
        self.condensed = condensed
        self.sort_mode = sort_mode
        self._validate_func_options()
        self.n_s = kwargs.get("n_s", 0.05)
        self.n_e = kwargs.get("n_e", 1.0)
        self.val_s = kwargs.get("val_s", 1.0)
        self.val_e = kwargs.get("val_e", 0.05)
        self.max_val = kwargs.get("max_val", None)
        self.stream = kwargs.get("stream", None)
        self.nnz = 0
        self.nnz_discarded = 0
        self.csr_form = False
        self.is_diassoc = False
        self._csr = None
        self.max_count = 0
        self.cap_indptr = capacity_indptr(n_samples, max_assocs, max_assocs_type, self.n_s,
                                          self.n_e, self.val_s, self.val_e, self.stream)

    def _validate_func_options(self):
        """MyML/MyML/EAC/sparse.py:109-138 (same errors)."""
        if self.condensed not in (True, False):
            raise TypeError("condensed must be boolean")
        if not isinstance(self.max_assocs, (int, np.integer)):
            raise TypeError("max_assocs must be an integer")
        if self.max_assocs <= 0:
            raise ValueError("max_assocs must be an integer above 0")
        if not isinstance(self.n_samples, (int, np.integer)):
            raise TypeError("number of samples must be an integer")
        if self.n_samples <= 0:
            raise ValueError("number of samples must be an integer above 0")
        if not issubclass(self.dtype, (np.integer, np.floating)):
            raise TypeError("dtype must be a NumPy integer or float type")
        sort_options = ("numpy", "normal", "simple", "surgical")
        if self.sort_mode not in sort_options:
            raise ValueError("sort_mode must be one of the following: {}".format(sort_options))
        max_assocs_options = ("constant", "linear")
        if self.max_assocs_type not in max_assocs_options:
            raise ValueError("max_assocs_type must be one of the following: {}".format(
                max_assocs_options))
        if self.max_assocs_type != "constant" and not self.condensed:
            raise ValueError("max_assocs_type must be \"constant\" if matrix is condensed")
        if not self.condensed:
            raise NotImplementedError("only the condensed co-association matrix (the EAC "
                                      "default) is built on the GPU")
        if np.dtype(self.dtype) != np.uint8:
            raise NotImplementedError("co-association counts are uint8 (the EAC default)")

    def update_ensemble(self, ensemble, progress=False, builder=None):
        """Accumulate all partitions (MyML/MyML/EAC/sparse.py:154-166)."""
        if builder is None:
            t = _lib.torch()
            if isinstance(ensemble, (np.ndarray, t.Tensor)):
                labels = ensemble
            else:
                labels = label_matrix_from_ensemble(ensemble, self.n_samples)
            builder = CoassocBuilder(labels, self.n_samples, stream=self.stream)
        ip, ind, dat, nnz, disc, mx = builder.build(self.cap_indptr)
        self.indptr, self.indices, self.data = ip, ind, dat
        self.nnz += nnz
        self.nnz_discarded += disc
        self.max_count = mx
        self.csr_form = True

    def _condense(self, keep_degree=False):
        """The GPU build writes the condensed CSR directly (rows back to back);
        nothing left to do (MyML/MyML/EAC/sparse.py:212-226)."""
        self.csr_form = True

    def make_diassoc(self, max_val=None):
        """data = max_val - data, max_val = max count + 1 by default
        (MyML/MyML/EAC/sparse.py:295-304)."""
        if max_val is None:
            max_val = self.max_val + 1 if self.max_val is not None else self.max_count + 1
        _lib.check(_lib.load().eacb_make_diassoc(_lib.ptr(self.data), self.nnz, int(max_val),
                                                 _lib.stream_handle(self.stream)), "diassoc")
        self.is_diassoc = True
        self._csr = None

    @property
    def csr(self):
        if self._csr is None:
            from scipy.sparse import csr_matrix
            self._csr = csr_matrix((self.data.cpu().numpy(), self.indices.cpu().numpy(),
                                    self.indptr.cpu().numpy()),
                                   shape=(self.n_samples, self.n_samples))
        return self._csr

    def tocsr(self, copy=False):
        return self.csr.copy() if copy else self.csr

    def todense(self):
        return self.csr.todense()
