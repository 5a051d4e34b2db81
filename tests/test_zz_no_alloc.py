"""The allocation-free scan entry point, through the C ABI.

eacb_scan_excl_i32_noalloc serves callers that cannot allocate device memory
while they run (fixed memory pools, real-time paths, plugins handed raw
buffers), so it keeps its scratch in a fixed device array instead of taking
a workspace.  Its outputs are checked against the oracle's restatement of the
reference's exclusive scan (int32 prefixes wrap like the reference's) and
against the regular entry point, on calls made back to back so that each
call starts from whatever the previous one left in the shared array.  This
file is collected last so that a failure here leaves every other test
already run.
"""
import ctypes

import numpy as np
import pytest

import oracle

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
    ws = torch.empty(max(1, L.eacb_scan_workspace_size(x.numel())), dtype=torch.uint8,
                     device=x.device)
    _lib.check(L.eacb_scan_excl_i32(_lib.ptr(x), _lib.ptr(out), x.numel(), init, _lib.ptr(tot),
                                    _lib.ptr(ws), ws.numel(), stream), "scan")
    return out, tot


def _noalloc(_lib, L, x, out, init, stream):
    import torch
    tot = torch.full((1,), -7, dtype=torch.int64, device=x.device)
    st = L.eacb_scan_excl_i32_noalloc(_lib.ptr(x), _lib.ptr(out), x.numel(), init, _lib.ptr(tot),
                                      stream)
    assert st == 0, _lib.status_string(st)
    return int(tot.item())


def test_noalloc_scan_matches_oracle_and_regular_twice():
    import torch
    assert torch.cuda.is_available()
    _lib, L = _bind()
    stream = _lib.stream_handle()
    rng = np.random.default_rng(77)
    # calls in a row with different sizes and inputs: each must not see
    # anything the one before left in the shared scratch
    for n, init in ((5_000_003, 11), (3_000_000, -4)):
        a = rng.integers(-1000, 100_000, n).astype(np.int32)   # int32 prefixes wrap
        ref, ref_total = oracle.exprefixsum(a, init=init)
        x = torch.from_numpy(a).cuda()
        out = torch.empty_like(x)
        total = _noalloc(_lib, L, x, out, init, stream)
        assert np.array_equal(out.cpu().numpy(), ref)
        assert total == ref_total == init + int(a.astype(np.int64).sum())
        reg, reg_total = _regular(_lib, L, x, init, stream)
        assert torch.equal(out, reg)
        assert total == int(reg_total.item())


def test_noalloc_scan_empty_and_unaligned():
    import torch
    assert torch.cuda.is_available()
    _lib, L = _bind()
    stream = _lib.stream_handle()
    # n == 0: nothing is written and the total is the initial value
    x = torch.zeros(4, dtype=torch.int32, device="cuda")
    assert _noalloc(_lib, L, x[:0], x[:0], 9, stream) == 9
    # views one element off a 16-byte boundary take the scalar-load path
    rng = np.random.default_rng(78)
    a = rng.integers(0, 1000, 1_000_001).astype(np.int32)
    base = torch.from_numpy(a).cuda()
    dst = torch.full((a.size,), 123, dtype=torch.int32, device="cuda")
    xin, xout = base[1:], dst[1:]
    assert xin.data_ptr() % 16 != 0 and xout.data_ptr() % 16 != 0
    ref, ref_total = oracle.exprefixsum(a[1:], init=3)
    assert _noalloc(_lib, L, xin, xout, 3, stream) == ref_total
    assert np.array_equal(xout.cpu().numpy(), ref)
    assert int(dst[0].item()) == 123                       # nothing written before the view
    # and once more in place, right after
    ref2, ref2_total = oracle.exprefixsum(a, init=0)
    assert _noalloc(_lib, L, base, base, 0, stream) == ref2_total
    assert np.array_equal(base.cpu().numpy(), ref2)


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
