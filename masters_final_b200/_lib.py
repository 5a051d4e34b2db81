"""ctypes binding of libeacb200.so (the C ABI declared in include/eacb200.h).

PyTorch is used only for device buffers and streams.  There is no fallback:
if the library or a CUDA device is missing, every entry point raises.
"""
import contextlib
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libeacb200.so")

U8, U16, I32, U32, F32 = 1, 2, 3, 4, 5
_DTYPE_CODE = {np.dtype(np.uint8): U8, np.dtype(np.uint16): U16, np.dtype(np.int32): I32,
               np.dtype(np.uint32): U32, np.dtype(np.float32): F32}

ERR_VALUE = -9
ERR_FIRST_OVERFLOW = -7
ERR_WORKSPACE = -2

_lib = None

class EACBError(RuntimeError):
    def __init__(self, status, where, cuda=None):
        self.status = status
        msg = "%s failed: %s (%d)" % (where, status_string(status), status)
        if status == -3:
            if cuda is None:
                f = ctypes.c_char_p()
                ln = ctypes.c_int(0)
                code = load().eacb_last_cuda_error(ctypes.byref(f), ctypes.byref(ln))
                cuda = (code, (f.value or b"").decode(), ln.value)
            msg += "; cudaError %d at %s:%d" % cuda
        super().__init__(msg)


def load():
    """Load the library (build it first if this checkout has none)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libeacb200.so is not built; run `python -m masters_final_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    p, i32, i64, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_size_t
    P64 = ctypes.POINTER(ctypes.c_int64)
    P32 = ctypes.POINTER(ctypes.c_int32)
    sigs = {
        "eacb_version": (ctypes.c_int, []),
        "eacb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "eacb_last_cuda_error": (ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p),
                                                ctypes.POINTER(ctypes.c_int)]),
        "eacb_workspace_status": (ctypes.c_int, [p, p]),
        "eacb_profile_enable": (None, [ctypes.c_int]),
        "eacb_profile_read": (None, [p, p, p, p]),
        "eacb_scan_workspace_size": (sz, [i64]),
        "eacb_scan_excl_i32": (ctypes.c_int, [p, p, i64, i64, p, p, sz, p]),
        "eacb_scan_excl_i32_i64": (ctypes.c_int, [p, p, i64, i64, p, p, sz, p]),
        "eacb_scan_excl_i64": (ctypes.c_int, [p, p, i64, i64, p, p, sz, p]),
        "eacb_tune_set": (ctypes.c_int, [ctypes.c_int, i64, i64, i64, i64, i64]),
        "eacb_tune_clear": (None, []),
        "eacb_tune_get": (i64, [ctypes.c_int, i64, i64, i64]),
        "eacb_debug_set_round_cap": (None, [ctypes.c_int]),
        "eacb_debug_set_round_team": (None, [ctypes.c_int]),
        "eacb_boruvka_workspace_size": (sz, [i32, i64]),
        "eacb_boruvka_mst": (ctypes.c_int, [p, p, ctypes.c_int, p, p, i32, i64, p, P64, p, sz, p]),
        "eacb_connected_components": (ctypes.c_int, [p, p, ctypes.c_int, p, p, i32, i64, p, P64,
                                                     p, sz, p]),
        "eacb_kmeans_workspace_size": (sz, [i32, i32, i32, i32]),
        "eacb_kmeans_ensemble": (ctypes.c_int, [p, i32, i32, i32, p, i32, p, i32, ctypes.c_float,
                                                i32, i32, p, p, p, p, p, p, sz, p]),
        "eacb_kmeans_label_workspace_size": (sz, [i32, i32, i32]),
        "eacb_kmeans_label": (ctypes.c_int, [p, i32, i32, p, i32, i32, p, p, p, sz, p]),
        "eacb_coassoc_workspace_size": (sz, [i32, i32, i32]),
        "eacb_coassoc_prepare": (ctypes.c_int, [p, i32, i32, i32, P64, p, sz, p]),
        "eacb_coassoc_count": (ctypes.c_int, [p, i32, i32, i32, p, p, P64, p, sz, p]),
        "eacb_capacity_workspace_size": (sz, [i32]),
        "eacb_capacity_linear": (ctypes.c_int, [i32, i64, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_double, p, p, sz, p]),
        "eacb_capacity_constant": (ctypes.c_int, [i32, i64, p, p]),
        "eacb_make_diassoc": (ctypes.c_int, [p, i64, i32, p]),
        "eacb_coassoc_fill": (ctypes.c_int, [p, i32, i32, i32, p, p, p, p, i32, P64, P32, p, sz,
                                             p]),
        "eacb_kmeans_label_fp32": (ctypes.c_int, [p, i32, i32, p, i32, p, p, p, sz, p]),
        "eacb_kmeans_label_bf16tc": (ctypes.c_int, [p, i32, i32, p, i32, p, p, p, sz, p]),
        "eacb_kmeans_centroids_workspace_size": (sz, [i32, i32, i32]),
        "eacb_kmeans_centroids": (ctypes.c_int, [p, i32, i32, p, p, i32, i32, p, p, sz, p]),
        "eacb_coassoc_build_workspace_size": (sz, [i32, i32, i32]),
        "eacb_coassoc_build": (ctypes.c_int, [p, i32, i32, i32, i32, i64, i32, p, p, p, i64, i32,
                                              P64, P64, P32, P64, p, sz, p]),
        "eacb_lifetime_cut_workspace_size": (sz, []),
        "eacb_lifetime_cut": (ctypes.c_int, [p, i64, i32, i32, i32, P64, P32, p, sz, p]),
        "eacb_relabel_canonical_workspace_size": (sz, [i32]),
        "eacb_relabel_canonical": (ctypes.c_int, [p, i32, p, P64, p, sz, p]),
        "eacb_batched_workspace_size": (sz, [p, i32, i32]),
        "eacb_batched_eac": (ctypes.c_int, [p, i32, p, i32, p, sz, p]),
        "eacb_final_clustering_workspace_size": (sz, [i32, i64]),
        "eacb_final_clustering": (ctypes.c_int, [p, p, p, i32, i64, i32, i32, p, P64, P32, p, sz,
                                                 p]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    if os.environ.get("EACB_TUNING", "1") != "0":
        apply_tuning()
    return L


# ---------------------------------------------------------------- tuning ---
TUNING_PATH = os.path.join(_HERE, "tuning.json")
TUNE_KNOBS = {"tc_ctas_per_sm": 0, "tc_buffers": 1, "co_count_ctas": 2, "co_fill_ctas": 3,
              "mst_phase1_permille": 4, "round_team": 5, "co_dense_ratio": 6}
_tuning = {"python": {}, "applied": False}


def apply_tuning(path=None):
    """Loads the autotuner's table (masters_final_b200/tuning.json by
    default) into the library's launch-shape table; entries the library
    does not know are refused.  Returns the number of entries loaded."""
    L = load()
    L.eacb_tune_clear()
    _tuning["python"] = {}
    _tuning["applied"] = False
    return _add_table(L, path or TUNING_PATH)


def _add_table(L, path):
    import json
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        table = json.load(f)
    n = 0
    for e in table.get("entries", []):
        knob = TUNE_KNOBS[e["knob"]]
        check(L.eacb_tune_set(knob, int(e["a"][0]), int(e["a"][1]), int(e["b"][0]),
                              int(e["b"][1]), int(e["value"])), "tuning table")
        n += 1
    _tuning["python"] = dict(table.get("python", {}))
    _tuning["applied"] = True
    return n


@contextlib.contextmanager
def forced(name, value):
    """Within the block the knob `name` takes `value` for every shape (an
    entry ahead of the loaded table); the table is reloaded afterwards."""
    L = load()
    was = _tuning["applied"]
    L.eacb_tune_clear()
    check(L.eacb_tune_set(TUNE_KNOBS[name], 0, 1 << 62, 0, 1 << 62, int(value)), "tuning table")
    if was:
        _add_table(L, TUNING_PATH)
    try:
        yield
    finally:
        if was:
            apply_tuning()
        else:
            clear_tuning()


def clear_tuning():
    """Back to the built-in launch shapes (the untuned configuration)."""
    load().eacb_tune_clear()
    _tuning["python"] = {}
    _tuning["applied"] = False


def tuned(name, default):
    """A host-side tuned setting (e.g. the batched worker count)."""
    return _tuning["python"].get(name, default)


class Instance(ctypes.Structure):
    """struct eacb_instance (include/eacb200.h)."""
    _fields_ = [("X", ctypes.c_void_p), ("k", ctypes.c_void_p), ("init", ctypes.c_void_p),
                ("labels", ctypes.c_void_p), ("n", ctypes.c_int32), ("d", ctypes.c_int32),
                ("P", ctypes.c_int32), ("kmax", ctypes.c_int32), ("n_fclusts", ctypes.c_int64),
                ("nnz", ctypes.c_int64), ("nnz_discarded", ctypes.c_int64),
                ("labels_valid", ctypes.c_int32), ("status", ctypes.c_int32),
                ("ms_ensemble", ctypes.c_float), ("ms_coassoc", ctypes.c_float),
                ("ms_final", ctypes.c_float), ("worker", ctypes.c_int32),
                ("cuda_error", ctypes.c_int32), ("cuda_line", ctypes.c_int32)]


class BatchOptions(ctypes.Structure):
    """struct eacb_batch_options (include/eacb200.h)."""
    _fields_ = [("max_iter", ctypes.c_int32), ("tol", ctypes.c_float),
                ("label_mode", ctypes.c_int32), ("centroid_mode", ctypes.c_int32),
                ("cap_mode", ctypes.c_int32), ("max_assocs_factor", ctypes.c_int32),
                ("n_s", ctypes.c_double), ("n_e", ctypes.c_double), ("val_s", ctypes.c_double),
                ("val_e", ctypes.c_double), ("n_clusters", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


def extend(sigs):
    """Register more signatures (used by modules that add entry points)."""
    L = load()
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def profile_enable(on=True):
    load().eacb_profile_enable(1 if on else 0)


def profile_read():
    """(launches, per-tag ms, per-tag algorithmic bytes, per-tag launch counts)."""
    launches = ctypes.c_int64(0)
    ms = (ctypes.c_double * 8)()
    by = (ctypes.c_double * 8)()
    cnt = (ctypes.c_int64 * 8)()
    load().eacb_profile_read(ctypes.byref(launches), ms, by, cnt)
    return int(launches.value), list(ms), list(by), list(cnt)


def status_string(s):
    return load().eacb_status_string(s).decode()


def check(status, where):
    if status != 0:
        raise EACBError(status, where)


def exported_symbols():
    """Names declared in include/eacb200.h (the C ABI)."""
    import re
    hdr = os.path.join(os.path.dirname(_HERE), "include", "eacb200.h")
    with open(hdr) as f:
        txt = f.read()
    decl = r"^(?:const\s+)?\w+\s*\*?\s*(eacb_\w+)\s*\("
    return sorted(set(re.findall(decl, txt, flags=re.MULTILINE)))


# --------------------------------------------------------------- devices ---
def torch():
    import torch as _t
    return _t


def device():
    t = torch()
    if not t.cuda.is_available():
        raise RuntimeError("masters_final_b200 needs a CUDA device (B200, sm_100a)")
    return t.device("cuda", t.cuda.current_device())


def stream_handle(stream=None):
    t = torch()
    s = stream if stream is not None else t.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def ptr(x):
    return ctypes.c_void_p(x.data_ptr()) if x is not None else None


def workspace(nbytes):
    t = torch()
    return t.empty(max(int(nbytes), 256), dtype=t.uint8, device=device())


def to_device(a, dtype=None):
    """numpy array or torch tensor -> contiguous CUDA tensor (no copy if
    already there with the right dtype).  A pinned host tensor is copied
    asynchronously on the current stream, which the library's calls use."""
    t = torch()
    if isinstance(a, t.Tensor):
        x = a
        if dtype is not None and x.dtype != dtype and x.is_cuda:
            x = x.to(dtype)
        if not x.is_cuda:
            pinned = x.is_pinned()
            x = x.to(device(), non_blocking=pinned)
            if dtype is not None and x.dtype != dtype:
                x = x.to(dtype)
        return x.contiguous()
    arr = np.ascontiguousarray(a)
    x = t.from_numpy(arr)
    if dtype is not None:
        x = x.to(dtype)
    return x.to(device(), non_blocking=False).contiguous()


def to_host(x):
    """CUDA tensor -> numpy array through a pinned host buffer (torch's
    caching host allocator): the copy runs at the link's speed instead of
    being staged through pageable memory, and the array is a view that
    keeps the buffer alive.  Copies on the current stream and waits for it
    (the library's calls have finished their own stream by then)."""
    t = torch()
    if x.numel() == 0:
        return np.empty(tuple(x.shape), dtype=np_dtype_of(x))
    h = t.empty(tuple(x.shape), dtype=x.dtype, pin_memory=True)
    h.copy_(x.contiguous(), non_blocking=True)
    t.cuda.current_stream(x.device).synchronize()
    return h.numpy()


def np_dtype_of(x):
    t = torch()
    if isinstance(x, t.Tensor):
        return np.dtype(str(x.dtype).replace("torch.", ""))
    return np.asarray(x).dtype


def dtype_code(x):
    d = np_dtype_of(x)
    if d not in _DTYPE_CODE:
        raise TypeError("unsupported weight dtype %s" % d)
    return _DTYPE_CODE[d]
