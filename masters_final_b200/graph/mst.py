"""Boruvka minimum spanning forest on the GPU.

Drop-in for MyML/MyML/graph/mst.py:417-564 (``boruvka_minho_gpu``).  Same
inputs (a symmetric CSR split into dest / weight / firstEdge / outDegree) and
the same return contract ``(mst_edge_ids int32, n_edges)``; the chosen edges
are those of the unique forest under the order (weight, min(u,v), max(u,v)).
"""
import ctypes

from .. import _lib


def _csr_args(dest, weight, firstEdge, outDegree):
    t = _lib.torch()
    d = _lib.to_device(dest, t.int32)
    w = _lib.to_device(weight)
    f = _lib.to_device(firstEdge, t.int32)
    o = _lib.to_device(outDegree, t.int32)
    return d, w, f, o


def boruvka_minho_gpu(dest, weight, firstEdge, outDegree, MAX_TPB=512, stream=None,
                      returnDevAry=False):
    """Minimum spanning forest.  Returns (mst, n_edges): mst holds input edge
    ids (int32, numpy unless returnDevAry) of the n_edges chosen edges.
    MAX_TPB is accepted for compatibility; launch shapes are fixed."""
    t = _lib.torch()
    d, w, f, o = _csr_args(dest, weight, firstEdge, outDegree)
    V = f.numel()
    E = d.numel()
    L = _lib.load()
    ws = _lib.workspace(L.eacb_boruvka_workspace_size(V, E))
    mst = t.empty(max(V - 1, 1), dtype=t.int32, device=d.device)
    n = ctypes.c_int64(0)
    _lib.check(L.eacb_boruvka_mst(_lib.ptr(d), _lib.ptr(w), _lib.dtype_code(w), _lib.ptr(f),
                                  _lib.ptr(o), V, E, _lib.ptr(mst), ctypes.byref(n),
                                  _lib.ptr(ws), ws.numel(), _lib.stream_handle(stream)),
               "boruvka_minho_gpu")
    n = int(n.value)
    if returnDevAry:
        return mst, n
    # V - 1 entries, the first n of them the forest (the reference's shape)
    return _lib.to_host(mst[:max(V - 1, 0)]), n


# The reference ships a CPU twin with the same contract
# (MyML/MyML/graph/mst.py:143-232); here both names run on the GPU.
boruvka_minho_seq = boruvka_minho_gpu
