"""The allocation-free scan entry point against the regular one.

eacb_scan_excl_i32_noalloc serves callers that cannot allocate device memory
while they run (fixed memory pools, real-time paths, plugins handed raw
buffers), so it keeps its scratch in a fixed device array instead of taking
a workspace.  This file is collected last so that a failure here leaves every
other test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind():
    from masters_final_b200 import _lib
    L = _lib.load()
    p, i64 = ctypes.c_void_p, ctypes.c_int64
    L.eacb_scan_excl_i32_noalloc.restype = ctypes.c_int
    L.eacb_scan_excl_i32_noalloc.argtypes = [p, p, i64, i64, p, p]
    return _lib, L


def _regular(_lib, L, x, init, stream):
    import torch
    out = torch.empty_like(x)
    tot = torch.empty(1, dtype=torch.int64, device=x.device)
    ws = torch.empty(L.eacb_scan_workspace_size(x.numel()), dtype=torch.uint8, device=x.device)
    _lib.check(L.eacb_scan_excl_i32(_lib.ptr(x), _lib.ptr(out), x.numel(), init, _lib.ptr(tot),
                                    _lib.ptr(ws), ws.numel(), stream), "scan")
    return out, tot


def test_noalloc_scan_matches_regular_twice():
    import torch
    assert torch.cuda.is_available()
    _lib, L = _bind()
    stream = _lib.stream_handle()
    rng = np.random.default_rng(77)
    # two calls in a row with different sizes and inputs: the second must not
    # see anything the first left in the shared scratch
    for n, init in ((5_000_003, 11), (3_000_000, -4)):
        a = rng.integers(-1000, 100_000, n).astype(np.int32)   # int32 prefixes wrap
        x = torch.from_numpy(a).cuda()
        ref, ref_tot = _regular(_lib, L, x, init, stream)
        out = torch.empty_like(x)
        tot = torch.empty(1, dtype=torch.int64, device=x.device)
        st = L.eacb_scan_excl_i32_noalloc(_lib.ptr(x), _lib.ptr(out), n, init, _lib.ptr(tot),
                                          stream)
        assert st == 0, _lib.status_string(st)
        assert torch.equal(out, ref)
        assert int(tot.item()) == int(ref_tot.item()) == init + int(a.astype(np.int64).sum())


def test_noalloc_scan_rejects_sizes_beyond_its_scratch():
    import torch
    assert torch.cuda.is_available()
    _lib, L = _bind()
    x = torch.zeros(16, dtype=torch.int32, device="cuda")
    tot = torch.empty(1, dtype=torch.int64, device="cuda")
    too_big = (1 << 28) + 1                      # EACB_SCAN_NOALLOC_MAX_N + 1
    st = L.eacb_scan_excl_i32_noalloc(_lib.ptr(x), _lib.ptr(x), too_big, 0, _lib.ptr(tot),
                                      _lib.stream_handle())
    assert _lib.status_string(st) == "EACB_ERR_WORKSPACE"
