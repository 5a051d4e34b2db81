"""Autotuner of the launch shapes (writes masters_final_b200/tuning.json).

    python -m masters_final_b200.tune [--out PATH] [--quick]

The reference fixes its launch shapes by hand (MyML/MyML/cluster/KMeans.py:
286-291 sizes its grid from a constant thread count); here each knob of the
library's tuning table (csrc/tune.cu) is timed over its candidates on the
shapes of the EAC workloads -- with CUDA events, after a warm-up, the best
of a few runs -- and the fastest candidate is written to a JSON table with
the timings that chose it.  The Python binding loads the table when the
library is loaded (EACB_TUNING=0 skips it), so every later call uses the
tuned shapes.

Knobs and the stage each one is timed on:
  tc_ctas_per_sm, tc_buffers   one batched K-Means fit of 4 partitions on the
                               tensor-core labeler (per dimension d and n;
                               1, 2 or 4 CTAs per SM)
  co_dense_ratio               the co-association build of a 20-partition
                               K-Means ensemble (per n); the streaming
                               passes' CTAs per SM keep their defaults
  mst_phase1_permille,         the Boruvka MST of the 16-NN graph of 1M points
  round_team (graph)
  round_team (EAC)             the final clustering of a co-association
                               matrix (single instances)
  batched_workers              one eac_batch call over 128 of the 512
                               datasets (host worker threads)
"""
import argparse
import ctypes
import itertools
import json
import os
import random
import time

import numpy as np

from . import _lib

# shapes of the EAC workloads: (name, n, d, mixture components, k range)
KMEANS_SHAPES = [
    ("eac_500k_16d", 500_000, 16, 50, (350, 711)),
    ("eac_2m_8d", 2_000_000, 8, 200, (700, 1401)),
    ("batched_small_32d", 12_000, 32, 10, (55, 110)),
    ("batched_small_2d", 12_000, 2, 10, (55, 110)),
]
COASSOC_SHAPES = [("eac_500k", 500_000, (350, 711)), ("eac_2m", 2_000_000, (700, 1401))]


def _best_ms(fn, reps=3, warm=1):
    t = _lib.torch()
    st = t.cuda.current_stream()
    for _ in range(warm):
        fn()
    best = float("inf")
    for _ in range(reps):
        a, b = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        a.record(st)
        fn()
        b.record(st)
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def _set(L, knob, a, b, value):
    _lib.check(L.eacb_tune_set(_lib.TUNE_KNOBS[knob], a[0], a[1], b[0], b[1], int(value)),
               "tuning table")


def _sweep(L, grid, run, fixed):
    """Times run() for every combination in grid (knob -> (a, b, values)),
    with the fixed entries first; returns (best combination, timings)."""
    names = list(grid)
    timings = []
    for combo in itertools.product(*(grid[k][2] for k in names)):
        L.eacb_tune_clear()
        for knob, a, b, v in fixed:
            _set(L, knob, a, b, v)
        for k, v in zip(names, combo):
            _set(L, k, grid[k][0], grid[k][1], v)
        timings.append((dict(zip(names, combo)), run()))
    best = min(timings, key=lambda x: x[1])[0]
    return best, [{"values": c, "ms": round(ms, 4)} for c, ms in timings]


def tune_kmeans(L, quick, out):
    from . import workloads as W
    from .cluster.KMeans import kmeans_ensemble
    t = _lib.torch()
    for name, n, d, comps, kr in KMEANS_SHAPES[:2] if quick else KMEANS_SHAPES:
        x = W.gaussian_mixture(n, d, comps, seed=1, sigma=1.0, center_range=20.0)
        X = t.from_numpy(x).cuda()
        rng = np.random.default_rng(2)
        ks = [int(k) for k in rng.integers(kr[0], kr[1], 4)]
        inits = [rng.choice(n, k, replace=False).tolist() for k in ks]
        a, b = (d, d), (n // 2, n * 2)
        best, timings = _sweep(L, {"tc_ctas_per_sm": (a, b, (1, 2, 4)), "tc_buffers": (a, b, (1, 2))},
                               lambda: _best_ms(lambda: kmeans_ensemble(
                                   X, ks, inits, max_iter=3, label_mode="bf16")), [])
        for k, v in best.items():
            out["entries"].append({"knob": k, "a": list(a), "b": list(b), "value": v,
                                   "shape": name, "timings": timings})
        del X


def tune_coassoc(L, quick, out):
    """The pair tiles' work ratio (co_dense_ratio) on the co-association of a
    20-partition K-Means ensemble of each workload's data (the choice only
    moves groups between two exact paths)."""
    import random as _random
    from . import workloads as W
    from .EAC.sparse import CoassocBuilder, capacity_indptr
    from .utils.partition import generate_ensemble_labels
    t = _lib.torch()
    for name, n, kr in COASSOC_SHAPES[:1] if quick else COASSOC_SHAPES:
        d, comps = (16, 50) if n <= 500_000 else (8, 200)
        x = W.gaussian_mixture(n, d, comps, seed=3, sigma=1.0, center_range=20.0)
        X = t.from_numpy(x).cuda()
        np.random.seed(3)
        _random.seed(3)
        Ld, _ = generate_ensemble_labels(X, list(kr), 20, 3, label_mode="bf16")
        del X
        a, b = (1, 255), (n // 2, n * 2)

        def run():
            bb = CoassocBuilder(Ld, n)
            cap = capacity_indptr(n, bb.max_cluster * 3)
            return _best_ms(lambda: bb.build(cap), reps=2)
        best, timings = _sweep(L, {"co_dense_ratio": (a, b, (4, 16, 64))}, run, [])
        for k, v in best.items():
            out["entries"].append({"knob": k, "a": list(a), "b": list(b), "value": v,
                                   "shape": name + " (20 K-Means partitions)", "timings": timings})
        del Ld
        t.cuda.empty_cache()


def tune_mst(L, quick, out):
    from . import workloads as W
    t = _lib.torch()
    indptr, dest, w = W.knn_graph(1_000_000, k=16, seed=2)
    V, E = indptr.size - 1, dest.size
    d = [t.from_numpy(a).cuda() for a in (dest, w, indptr[:-1].astype(np.int32),
                                           np.diff(indptr).astype(np.int32))]
    ws = t.empty(L.eacb_boruvka_workspace_size(V, E), dtype=t.uint8, device="cuda")
    mst = t.empty(V, dtype=t.int32, device="cuda")
    nm = ctypes.c_int64(0)
    sh = _lib.stream_handle()

    def run():
        def step():
            _lib.check(L.eacb_boruvka_mst(_lib.ptr(d[0]), _lib.ptr(d[1]), _lib.U8, _lib.ptr(d[2]),
                                          _lib.ptr(d[3]), V, E, _lib.ptr(mst), ctypes.byref(nm),
                                          _lib.ptr(ws), ws.numel(), sh), "mst")
        return _best_ms(step, reps=5, warm=2)
    a, b = (0, 0), (V // 4, V * 4)
    grid = {"mst_phase1_permille": (a, b, (125, 250, 375) if quick else (125, 188, 250, 375, 500)),
            "round_team": (a, b, (0, 74))}
    best, timings = _sweep(L, grid, run, [])
    for k, v in best.items():
        out["entries"].append({"knob": k, "a": list(a), "b": list(b), "value": v,
                               "shape": "knn16_1M graph MST", "timings": timings})


def tune_batched(L, quick, out):
    from . import workloads as W
    from .EAC.batched import draw_instance_params, eac_batch, k_range_rule1
    t = _lib.torch()
    xs = W.batched_instances(512, seed=0)[::4]
    ps = [draw_instance_params(x.shape[0], k_range_rule1(x.shape[0]), 50, i)
          for i, x in enumerate(xs)]
    Xd = [t.from_numpy(x).cuda() for x in xs]
    timings = []
    for nw in ((16, 32) if quick else (16, 24, 32, 48, 64)):
        eac_batch(Xd, params=ps, n_workers=nw, return_device=True)
        t.cuda.synchronize()
        t0 = time.perf_counter()
        eac_batch(Xd, params=ps, n_workers=nw, return_device=True)
        t.cuda.synchronize()
        timings.append({"values": {"batched_workers": nw},
                        "ms": round(1e3 * (time.perf_counter() - t0), 2)})
    best = min(timings, key=lambda x: x["ms"])["values"]["batched_workers"]
    out["python"]["batched_workers"] = best
    out["python_timings"] = {"batched_workers": timings,
                             "shape": "128 of the 512 batched datasets"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=_lib.TUNING_PATH)
    ap.add_argument("--quick", action="store_true", help="fewer shapes and candidates")
    args = ap.parse_args()
    os.environ["EACB_TUNING"] = "0"
    t = _lib.torch()
    L = _lib.load()
    random.seed(0)
    out = {"version": 1, "device": t.cuda.get_device_name(), "entries": [], "python": {},
           "how": "best of repeated CUDA-event timings of each candidate combination after a "
                  "warm-up (python knobs: host wall clock of one call after a warm-up call)"}
    for step in (tune_kmeans, tune_coassoc, tune_mst, tune_batched):
        step(L, args.quick, out)
        L.eacb_tune_clear()
        t.cuda.empty_cache()
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", args.out, len(out["entries"]), "entries;", out["python"])


if __name__ == "__main__":
    main()
