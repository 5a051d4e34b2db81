"""Connected components on the GPU.

Drop-in for MyML/MyML/graph/connected_components.py:176-314
(``connected_comps_gpu``) and its CPU twin ``connected_comps_seq`` (:46-137):
the labels are the reference's own numbering (Boruvka contraction picking the
minimum (weight, destination) out-edge, renumbering supervertices in root
order each round).
"""
import ctypes

import numpy as np

from .. import _lib
from .mst import _csr_args


def connected_comps_gpu(dest, weight, firstEdge, outDegree, MAX_TPB=512, stream=None,
                        returnDevAry=False):
    """Component label of every vertex (int32)."""
    t = _lib.torch()
    d, w, f, o = _csr_args(dest, weight, firstEdge, outDegree)
    V = f.numel()
    E = d.numel()
    L = _lib.load()
    ws = _lib.workspace(L.eacb_boruvka_workspace_size(V, E))
    labels = t.empty(V, dtype=t.int32, device=d.device)
    nc = ctypes.c_int64(0)
    _lib.check(L.eacb_connected_components(_lib.ptr(d), _lib.ptr(w), _lib.dtype_code(w),
                                           _lib.ptr(f), _lib.ptr(o), V, E, _lib.ptr(labels),
                                           ctypes.byref(nc), _lib.ptr(ws), ws.numel(),
                                           _lib.stream_handle(stream)),
               "connected_comps_gpu")
    if returnDevAry:
        return labels
    return _lib.to_host(labels)


connected_comps_seq = connected_comps_gpu
