"""Batched EAC: the reference's per-dataset experiment loop as one call.

The reference's experiment drivers (experiments/study_kmin.py:398-587) run,
for each dataset, generateEnsemble (MyML/MyML/utils/partition.py:88-124),
EAC.buildMatrix (MyML/MyML/EAC/eac.py:115-140) and EAC.finalClustering
(:142-179), one dataset after another.  ``eac_batch`` takes the whole list:
the host random draws of every instance are made exactly as the reference
makes them (legacy np.random for k, Python random.sample for the initial
centroids, seeded per instance), and libeacb200's ``eacb_batched_eac`` runs
all instances on the GPU with several in flight at once.
"""
import ctypes
import math
import random

import numpy as np

from .. import _lib
from ..cluster.KMeans import _CENTROID, _LABEL
from ..utils.partition import draw_ensemble_params


def k_range_rule1(n):
    """MyML/MyML/EAC/rules.py:17-22 (rule1): [ceil(sqrt(n)/2), ceil(sqrt(n))]."""
    return [int(math.ceil(np.sqrt(n) / 2)), int(math.ceil(np.sqrt(n)))]


class BatchResult:
    """Per-instance outcome: ``labels`` (numpy int32, numbered by smallest
    member; all zeros for a single cluster), ``n_fclusts``, ``nnz``,
    ``nnz_discarded``, ``labels_valid`` and ``status`` (0 = ok)."""

    def __init__(self, labels, n_fclusts, nnz, nnz_discarded, labels_valid, status,
                 ms_stages=None, worker=-1):
        self.labels = labels
        self.n_fclusts = n_fclusts
        self.nnz = nnz
        self.nnz_discarded = nnz_discarded
        self.labels_valid = labels_valid
        self.status = status
        self.ms_stages = ms_stages   # (ensemble, co-association, final) host ms on its worker
        self.worker = worker


def draw_instance_params(n, k_range, n_partitions, seed):
    """k per partition and initial samples of one instance, as the reference
    draws them after ``np.random.seed(seed); random.seed(seed)``."""
    np.random.seed(seed)
    random.seed(seed)
    return draw_ensemble_params(n, list(k_range), n_partitions)


def eac_batch(datasets, n_partitions=50, k_ranges=None, seeds=None, iters=3, tol=1e-4,
              label_mode="bf16", centroid_mode="numba", max_assocs_factor=3,
              max_assocs_type="linear", n_clusters=0, n_workers=None, arena_bytes=None,
              params=None, return_device=False, stream=None):
    """Run EAC on every dataset of ``datasets`` (list of (n_i, d_i) float32
    arrays, numpy or CUDA tensors; d_i <= 32).

    k_ranges: per-instance [kmin, kmax) (kmax exclusive, as generateEnsemble
    draws it); default ``k_range_rule1(n_i)``.  seeds: per-instance seed of
    the host draws (default: the instance index).  params: optional
    precomputed per-instance (ks, inits) lists, which replace the draws.
    arena_bytes: device memory for the count-dependent arrays of the
    instances in flight (default: half of the free device memory).
    Returns a list of BatchResult; raises EACBError if any instance failed
    (the results keep every instance's own status)."""
    t = _lib.torch()
    L = _lib.load()
    dev = _lib.device()
    m = len(datasets)
    if m == 0:
        return []
    if n_workers is None:
        n_workers = int(_lib.tuned("batched_workers", 16))
    if max_assocs_type not in ("linear", "constant"):
        raise ValueError("max_assocs_type must be 'linear' or 'constant'")
    if n_clusters < 0:
        raise ValueError("n_clusters must be >= 0")
    X = [_lib.to_device(x, t.float32) for x in datasets]
    ns = [int(x.shape[0]) for x in X]
    if params is None:
        params = []
        for i in range(m):
            kr = k_ranges[i] if k_ranges is not None else k_range_rule1(ns[i])
            sd = seeds[i] if seeds is not None else i
            params.append(draw_instance_params(ns[i], kr, n_partitions, sd))
    inst = (_lib.Instance * m)()
    keep = []
    for i in range(m):
        ks, inits = params[i]
        P = len(ks)
        kmax = int(max(ks))
        init = np.zeros((P, kmax), dtype=np.int32)
        for p, idx in enumerate(inits):
            init[p, :len(idx)] = idx
        k_d = t.tensor(np.asarray(ks, dtype=np.int32), device=dev)
        init_d = t.from_numpy(init).to(dev)
        lab = t.empty(ns[i], dtype=t.int32, device=dev)
        keep.append((k_d, init_d, lab))
        it = inst[i]
        it.X, it.k, it.init, it.labels = (X[i].data_ptr(), k_d.data_ptr(), init_d.data_ptr(),
                                          lab.data_ptr())
        it.n, it.d, it.P, it.kmax = ns[i], int(X[i].shape[1]), P, kmax
    opt = _lib.BatchOptions()
    opt.max_iter = int(iters)
    opt.tol = float(np.float32(tol))
    opt.label_mode = _LABEL[label_mode]
    opt.centroid_mode = _CENTROID[centroid_mode]
    opt.cap_mode = 0 if max_assocs_type == "linear" else 1
    opt.max_assocs_factor = int(max_assocs_factor)
    opt.n_s, opt.n_e, opt.val_s, opt.val_e = 0.05, 1.0, 1.0, 0.05
    opt.n_clusters = int(n_clusters)
    fixed = L.eacb_batched_workspace_size(inst, m, int(n_workers))
    if arena_bytes is None:
        free, _ = t.cuda.mem_get_info(dev)
        arena_bytes = max(free // 2 - fixed, 1 << 28)
    ws = t.empty(int(fixed + arena_bytes), dtype=t.uint8, device=dev)
    st = L.eacb_batched_eac(inst, m, ctypes.byref(opt), int(n_workers), _lib.ptr(ws), ws.numel(),
                            _lib.stream_handle(stream))
    out = []
    for i in range(m):
        it = inst[i]
        lab = keep[i][2] if return_device else keep[i][2].cpu().numpy()
        out.append(BatchResult(lab, int(it.n_fclusts), int(it.nnz), int(it.nnz_discarded),
                               int(it.labels_valid), int(it.status),
                               (float(it.ms_ensemble), float(it.ms_coassoc), float(it.ms_final)),
                               int(it.worker)))
    del ws
    if st != 0:
        first = next(inst[i] for i in range(m) if inst[i].status == st)
        err = _lib.EACBError(st, "batched eac",
                             (int(first.cuda_error), "batched instance", int(first.cuda_line)))
        err.results = out
        raise err
    return out


def instance_cost(n, d, P, kmax):
    """Relative GPU cost of one instance: co-association visits ~ P n (n / k)
    plus the ensemble's P n k d distance work."""
    k = max(int(kmax), 1)
    return float(P) * n * (n / k) + float(P) * n * k * d / 64.0


def shard_instances(costs, world):
    """Deterministic longest-processing-time assignment of instances to
    `world` ranks: returns one ascending index list per rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(o) for o in out]


def eac_batch_distributed(datasets, n_partitions=50, k_ranges=None, seeds=None, group=None,
                          runner=None, **kw):
    """eac_batch over the ranks of a torch.distributed process group: every
    rank receives the whole dataset list, runs its share (balanced by
    instance_cost, no data-path collective) on its own GPU, and the results
    are exchanged once at the end (all_gather_object), so every rank returns
    the full list in input order.  The host draws of instance i use seed
    seeds[i] (default i) whichever rank runs it, so results equal a
    single-GPU call."""
    import torch.distributed as dist
    run = runner or eac_batch
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    m = len(datasets)
    ns = [int(x.shape[0]) for x in datasets]
    kr = [k_ranges[i] if k_ranges is not None else k_range_rule1(ns[i]) for i in range(m)]
    sd = [seeds[i] if seeds is not None else i for i in range(m)]
    costs = [instance_cost(ns[i], int(datasets[i].shape[1]), n_partitions, kr[i][1])
             for i in range(m)]
    mine = shard_instances(costs, world)[rank]
    params = [draw_instance_params(ns[i], kr[i], n_partitions, sd[i]) for i in mine]
    kw["return_device"] = False              # results travel between ranks as numpy
    status = 0
    res = []
    if mine:
        try:
            res = run([datasets[i] for i in mine], n_partitions=n_partitions, params=params, **kw)
        except _lib.EACBError as e:          # every rank still joins the exchange
            status = e.status
            res = getattr(e, "results", [])
    local = (status, [(i, r) for i, r in zip(mine, res)])
    gathered = [None] * world
    dist.all_gather_object(gathered, local, group=group)
    out = [None] * m
    first_err = 0
    for st, part in gathered:
        first_err = first_err or st
        for i, r in part:
            out[i] = r
    if first_err:
        err = _lib.EACBError(first_err, "distributed batched eac", (0, "batched instance", 0))
        err.results = out
        raise err
    return out
