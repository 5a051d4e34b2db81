"""Exclusive prefix sums on the GPU.

Drop-in for MyML/MyML/utils/scan.py: ``scan_gpu`` (:144-249) and the CPU
helpers ``exprefixsumNumba`` (:42-53) / ``exprefixsumNumbaSingle`` (:57-72),
all computed by the single-pass decoupled look-back scan of libeacb200.
"""
import numpy as np

from .. import _lib


def _scan(x_dev, out_dev, init, stream=None):
    t = _lib.torch()
    n = x_dev.numel()
    L = _lib.load()
    ws = _lib.workspace(L.eacb_scan_workspace_size(n))
    total = t.empty(1, dtype=t.int64, device=x_dev.device)
    if x_dev.dtype == t.int32 and out_dev.dtype == t.int32:
        f = L.eacb_scan_excl_i32
    elif x_dev.dtype == t.int32 and out_dev.dtype == t.int64:
        f = L.eacb_scan_excl_i32_i64
    elif x_dev.dtype == t.int64 and out_dev.dtype == t.int64:
        f = L.eacb_scan_excl_i64
    else:
        raise NotImplementedError("non integer arrays are not supported")
    _lib.check(f(_lib.ptr(x_dev), _lib.ptr(out_dev), n, int(init), _lib.ptr(total),
                 _lib.ptr(ws), ws.numel(), _lib.stream_handle(stream)), "scan")
    return total, ws


def scan_gpu(in_ary, MAX_TPB=512, stream=0):
    """In-place exclusive scan of an integer array.  For a numpy input the
    array is updated and the total returned as a Python int; for a CUDA
    tensor the tensor is updated and a 1-element device tensor returned
    (MyML/MyML/utils/scan.py:144-249).  MAX_TPB is accepted for
    compatibility; tile shapes are fixed by the kernel."""
    t = _lib.torch()
    if isinstance(in_ary, np.ndarray):
        if not np.issubdtype(in_ary.dtype, np.integer):
            raise NotImplementedError("non integer arrays are not supported")
        d = _lib.to_device(in_ary)
        total, ws = _scan(d, d, 0)
        in_ary[...] = d.cpu().numpy()
        _lib.check(_lib.load().eacb_workspace_status(_lib.ptr(ws), _lib.stream_handle()), "scan")
        return int(total.item())
    if isinstance(in_ary, t.Tensor) and in_ary.is_cuda:
        if in_ary.dtype not in (t.int32, t.int64):
            raise NotImplementedError("non integer arrays are not supported")
        total, ws = _scan(in_ary, in_ary, 0)
        return total
    raise TypeError("input array must be a numpy array or a CUDA tensor")


def exprefixsumNumba(in_ary, out_ary, init=0):
    """out_ary[i] = init + sum(in_ary[:i]); returns the total
    (MyML/MyML/utils/scan.py:42-53).  int32 outputs wrap like the reference."""
    t = _lib.torch()
    if isinstance(in_ary, t.Tensor) and in_ary.is_cuda:
        total, ws = _scan(in_ary, out_ary, init)
        _lib.check(_lib.load().eacb_workspace_status(_lib.ptr(ws), _lib.stream_handle()), "scan")
        return int(total.item())
    x = _lib.to_device(in_ary)
    o = t.empty(x.numel(), dtype=getattr(t, _lib.np_dtype_of(out_ary).name), device=x.device)
    total, ws = _scan(x, o, init)
    _to_host(o, out_ary)
    _lib.check(_lib.load().eacb_workspace_status(_lib.ptr(ws), _lib.stream_handle()), "scan")
    return int(total.item())


def _to_host(dev, out):
    """Copies a device result into the caller's host array (numpy, or a torch
    CPU tensor -- pinned ones are written directly by the copy engine)."""
    t = _lib.torch()
    if isinstance(out, t.Tensor):
        out.copy_(dev.view(out.shape))
    else:
        out[...] = dev.cpu().numpy().reshape(out.shape)


def exprefixsumNumbaSingle(in_ary, init=0):
    """In-place exclusive scan with an initial value; returns the total
    (MyML/MyML/utils/scan.py:57-72)."""
    t = _lib.torch()
    if isinstance(in_ary, t.Tensor) and in_ary.is_cuda:
        total, ws = _scan(in_ary, in_ary, init)
        return int(total.item())
    x = _lib.to_device(in_ary)
    total, ws = _scan(x, x, init)
    _to_host(x, in_ary)
    _lib.check(_lib.load().eacb_workspace_status(_lib.ptr(ws), _lib.stream_handle()), "scan")
    return int(total.item())
