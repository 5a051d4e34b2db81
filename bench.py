#!/usr/bin/env python
"""Benchmark of the EAC hot path on B200.

Default workload: Boruvka minimum spanning forest of the 16-nearest-neighbour
graph of 1,000,000 uniform 3-D points (symmetrised, duplicates merged,
8,960,895 undirected edges with uint8 weights uniform in [1, 255], int32
indices).  Metric: MST edges/s = undirected input edges / MST time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1).  The forest does not shard: every
rank solves its own replica (replicas only, weak scaling) and `value` is the
edges of all replicas over the slowest rank's time.  `--impl reference` times
the reference's CPU algorithm (the oracle's C restatement of
boruvka_minho_seq) on the host cores instead.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_VERTICES = 1_000_000
KNN = 16
SEED = 2
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--no-eac", action="store_true",
                    help="skip the EAC end-to-end measurements added to the line")
    ap.add_argument("--no-graph", action="store_true",
                    help="skip the connected-components and scan measurements added to the line")
    ap.add_argument("--case", choices=sorted(CASES),
                    help="run one small named workload and exit (the cases the ncu summaries "
                         "under profiles/ were captured on)")
    return ap.parse_args()


def workload_config(n_edges):
    return {"workload": "boruvka_mst_knn16_1M",
            "graph": "16-NN of 1,000,000 uniform 3-D points, symmetrised",
            "n_vertices": N_VERTICES, "undirected_edges": int(n_edges),
            "directed_entries": int(2 * n_edges), "weights": "uint8 uniform [1,255]",
            "indices": "int32", "l2": "flushed (256 MiB write) between timed steps"}


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        # raw samples (the summary goes into the JSON line)
        self.out = os.path.join(os.environ.get("EACB_CLOCKS_DIR", tempfile.gettempdir()),
                                "clocks_bench_%d.csv" % index)

    def __enter__(self):
        os.makedirs(os.path.dirname(self.out), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.out, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index),
                                          "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        # the timed region is short (milliseconds): it starts only once the
        # sampler has written its first line
        self.lines0 = self._wait_lines(1, 5.0)
        return self

    def _lines(self):
        try:
            with open(self.out) as f:
                return sum(1 for _ in f)
        except OSError:
            return 0

    def _wait_lines(self, at_least, timeout_s):
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < timeout_s:
            self.f.flush()
            k = self._lines()
            if k >= at_least:
                return k
            time.sleep(0.005)
        return self._lines()

    def __exit__(self, *a):
        if self.proc is not None:
            # one more sample after the region, so that it is bracketed
            self._wait_lines(self.lines0 + 1, 2.0)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.out):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.out) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax.append(float(p[2]))
                except ValueError:
                    continue
                for name, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# kernels whose roofline the bench reports: (library profiling tag, name,
# algorithmic bytes per launch)
ROOF_KERNELS = [
    (0, "k_rounds (every Boruvka round of a weight phase in one persistent kernel)",
     "per round: 16 B per edge word (the word and its two endpoints' parents) + 8 B per "
     "surviving word written back + 20 B per active root (list entry, selection slot, "
     "successor, parent)"),
    (4, "k_phase_csr (weight-phase edge build + first min-edge selection)",
     "12 B per vertex (row extent, label) + 5 B per CSR entry (dest, uint8 weight) "
     "+ 8 B per edge word written"),
]


def profiled_traffic(kernel):
    """DRAM bytes per launch of `kernel` from its committed ncu summary
    (profiles/<kernel>_knn16_1M.md; None when there is none)."""
    name = {"k_rounds": "boruvka_rounds", "k_phase_csr": "boruvka_phase_csr"}.get(kernel)
    p = os.path.join(ROOT, "profiles", "%s_knn16_1M.md" % name) if name else ""
    if not p or not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    return None


def cpu_baseline(indptr, dest, w, n_edges, budget_s=12.0):
    import oracle
    times = []
    t_end = time.perf_counter() + budget_s
    while True:
        t0 = time.perf_counter()
        oracle.boruvka_seq(indptr, dest, w)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() > t_end or len(times) >= 10:
            break
    t = statistics.median(times)
    return {"value": n_edges / t, "unit": "edges/s", "cores": 1, "kind": "port",
            "sample": "full graph, %d runs of the oracle's C restatement of "
                      "boruvka_minho_seq (single-threaded, like the reference), median" % len(times)}


def reference_threads():
    """Host threads for the reference arm: every core this process may use,
    bounded so that the concurrent copies (~0.4 GB each) fit in half of the
    available memory."""
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    try:
        import psutil
        mem_cap = int(psutil.virtual_memory().available * 0.5 // (400 << 20))
    except ImportError:
        mem_cap = cores
    return max(1, min(cores or 1, mem_cap, 64))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from concurrent.futures import ThreadPoolExecutor
    from masters_final_b200 import workloads as W
    indptr, dest, w = W.knn_graph(N_VERTICES, k=KNN, seed=SEED)
    n_edges = dest.size // 2
    import oracle
    run = oracle.boruvka_seq_runner(indptr, dest, w)
    # the reference's Boruvka is sequential: one graph cannot use more than
    # one core, so every host thread runs its own copy of the graph and the
    # throughput is all copies' edges over the wall time of a step
    threads = reference_threads()
    times = []
    with ThreadPoolExecutor(threads) as ex:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            done = list(ex.map(lambda _: run(), range(threads)))
            dt = time.perf_counter() - t0
            assert all(x == done[0] for x in done)
            if i >= args.warmup:
                times.append(dt)
    tot = sum(times)
    val = threads * n_edges * len(times) / tot
    line = {"metric": "MST edges/s", "value": val, "unit": "edges/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * tot / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": workload_config(n_edges),
            "cpu_baseline": {"value": val, "unit": "edges/s", "cores": threads, "kind": "port",
                             "sample": "per step, %d concurrent copies of the full graph, one per "
                                       "host thread; the oracle's C restatement of "
                                       "boruvka_minho_seq (sequential, like the reference)"
                                       % threads},
            "e2e": {"value": val, "unit": "edges/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from masters_final_b200 import _lib
    from masters_final_b200 import workloads as W
    from masters_final_b200.graph.mst import boruvka_minho_gpu
    import ctypes

    indptr, dest, w = W.knn_graph(N_VERTICES, k=KNN, seed=SEED)
    n_edges = dest.size // 2
    first = indptr[:-1].astype(np.int32)
    deg = np.diff(indptr).astype(np.int32)
    dev = torch.device("cuda", local)
    d_dest = torch.from_numpy(dest).to(dev)
    d_w = torch.from_numpy(w).to(dev)
    d_first = torch.from_numpy(first).to(dev)
    d_deg = torch.from_numpy(deg).to(dev)
    L = _lib.load()
    V, E = N_VERTICES, dest.size
    ws = torch.empty(L.eacb_boruvka_workspace_size(V, E), dtype=torch.uint8, device=dev)
    mst = torch.empty(V, dtype=torch.int32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    nm = ctypes.c_int64(0)

    def step():
        _lib.check(L.eacb_boruvka_mst(_lib.ptr(d_dest), _lib.ptr(d_w), _lib.U8, _lib.ptr(d_first),
                                      _lib.ptr(d_deg), V, E, _lib.ptr(mst), ctypes.byref(nm),
                                      _lib.ptr(ws), ws.numel(), sh), "boruvka")

    def barrier():
        if world > 1:
            dist.all_reduce(torch.zeros(1, device=dev))
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    # ---- device-resident timed region ----
    barrier()
    _lib.profile_enable(False)          # clears the launch counter
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.fill_(i & 255)
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        barrier()
    launches = _lib.profile_read()[0]
    assert nm.value == V - 1
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    # ---- kernel roofline: a second pass with per-launch CUDA events ----
    # (profiling synchronizes after each timed launch, so it stays out of the
    # timed region above)
    _lib.profile_enable(True)
    p_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            for _ in range(args.steps)]
    for i in range(args.steps):
        flush.fill_(i & 255)
        p_ev[i][0].record(stream)
        step()
        p_ev[i][1].record(stream)
    torch.cuda.synchronize()
    _, pms, pbytes, pcount = _lib.profile_read()
    _lib.profile_enable(False)
    p_ms = sum(a.elapsed_time(b) for a, b in p_ev)
    t = torch.tensor([t_ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t_ms = float(t.item())
    value = world * n_edges * args.steps / (t_ms / 1000.0)

    # ---- end to end through the public API, host buffers (pinned) ----
    if args.no_e2e:
        e_ms = float("nan")
    h_dest = torch.from_numpy(dest).pin_memory()
    h_w = torch.from_numpy(w).pin_memory()
    h_first = torch.from_numpy(first).pin_memory()
    h_deg = torch.from_numpy(deg).pin_memory()
    if not args.no_e2e:
        boruvka_minho_gpu(h_dest, h_w, h_first, h_deg)      # warm
        barrier()
        e_ms = 0.0
    for i in range(0 if args.no_e2e else args.steps):
        flush.fill_(i & 255)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out, n = boruvka_minho_gpu(h_dest, h_w, h_first, h_deg)
        b.record(stream)
        b.synchronize()
        e_ms += a.elapsed_time(b)
        assert n == V - 1
    t = torch.tensor([e_ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e_ms = float(t.item())
    e2e = {"value": world * n_edges * args.steps / (e_ms / 1000.0), "unit": "edges/s",
           "h2d_bytes_per_step": int(dest.nbytes + w.nbytes + first.nbytes + deg.nbytes),
           "d2h_bytes_per_step": int(4 * (V - 1))}

    sharded = None
    if world > 1 and not args.no_eac:
        sharded = eac_batched_sharded_measurement(torch, dist, world)
    graph = None
    if world == 1 and not args.no_graph:
        graph = {"cc_knn16_1M": cc_measurement(torch, (indptr, dest, w, d_dest, d_w, d_first,
                                                         d_deg, ws), flush, args.steps),
                 "scan_64m": scan_measurement(torch, flush, measured_peak()[0], args.steps)}

    if rank == 0:
        peak, peak_kind = measured_peak()
        kernels = []
        for tag, name, algo in ROOF_KERNELS:
            if pms[tag] <= 0 or pcount[tag] == 0:
                continue
            achieved = (pbytes[tag] / (pms[tag] / 1000.0)) / 1e9
            kernels.append({"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                            "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                            "traffic": profiled_traffic(name.split()[0]),
                            "launches": int(pcount[tag]),
                            "ms_per_step": pms[tag] / args.steps,
                            "ms_share_of_step": pms[tag] / p_ms if p_ms else None,
                            "profiled_ms_per_step": p_ms / args.steps,
                            "algorithmic_bytes": algo})
        # the roofline object describes the kernel with the largest share
        roof = max(kernels, key=lambda k: k["ms_per_step"]) if kernels else None
        line = {"metric": "MST edges/s", "value": value, "unit": "edges/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u8", "data": "synthetic", "config": workload_config(n_edges),
                "e2e": e2e, "roofline": roof, "roofline_kernels": kernels,
                "gpu_launches": int(launches),
                "clocks": clk.summary()}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(indptr, dest, w, n_edges)
        if graph is not None:
            line["graph"] = graph
        if world == 1 and not args.no_eac:
            line["eac"] = eac_measurements(args)
        if sharded is not None:
            line["eac_batched_sharded"] = sharded
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ graph --
def _timed(torch, fn, steps, warm, flush):
    """Median CUDA-event milliseconds of fn() on the current stream, L2 flushed
    (a 256 MiB write) before each timed call."""
    st = torch.cuda.current_stream()
    for _ in range(warm):
        fn()
    ms = []
    for i in range(steps):
        flush.fill_(i & 255)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        fn()
        b.record(st)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    return statistics.median(ms)


def cc_measurement(torch, graph, flush, steps):
    """Connected components of the 16-NN graph (the reference's numbering):
    undirected edges/s device-resident, and end to end through
    connected_comps_gpu with pinned host buffers; CPU: the oracle's C
    restatement of the reference's Boruvka rounds, which connected_comps_seq
    runs with its labels tracked (one core)."""
    import ctypes
    import oracle
    from masters_final_b200 import _lib
    from masters_final_b200.graph.connected_components import connected_comps_gpu
    indptr, dest, w, d_dest, d_w, d_first, d_deg, ws = graph
    L = _lib.load()
    V, E = indptr.size - 1, dest.size
    n_edges = E // 2
    labels = torch.empty(V, dtype=torch.int32, device="cuda")
    nc = ctypes.c_int64(0)
    sh = _lib.stream_handle()

    def step():
        _lib.check(L.eacb_connected_components(_lib.ptr(d_dest), _lib.ptr(d_w), _lib.U8,
                                               _lib.ptr(d_first), _lib.ptr(d_deg), V, E,
                                               _lib.ptr(labels), ctypes.byref(nc), _lib.ptr(ws),
                                               ws.numel(), sh), "connected components")
    ms = _timed(torch, step, steps, 3, flush)
    h = [torch.from_numpy(a).pin_memory() for a in
         (dest, w, indptr[:-1].astype(np.int32), np.diff(indptr).astype(np.int32))]
    e_ms = _timed(torch, lambda: connected_comps_gpu(*h), max(3, steps // 2), 2, flush)
    # cpu_baseline leg: the oracle, timed
    t0 = time.perf_counter()
    oracle.boruvka_seq(indptr, dest, w)
    cpu_s = time.perf_counter() - t0
    return {"metric": "CC edges/s", "value": n_edges / (ms / 1e3), "unit": "edges/s",
            "ms": ms, "n_components": int(nc.value),
            "e2e": {"value": n_edges / (e_ms / 1e3), "unit": "edges/s", "ms": e_ms,
                    "h2d_bytes_per_step": int(sum(x.numel() * x.element_size() for x in h)),
                    "d2h_bytes_per_step": int(4 * V)},
            "cpu_baseline": {"value": n_edges / cpu_s, "unit": "edges/s", "cores": 1,
                             "kind": "port", "sample": "full graph, one run of the oracle's C "
                             "restatement of the reference's Boruvka rounds (the rounds "
                             "connected_comps_seq runs, labels tracked)"},
            "config": {"workload": "cc_knn16_1M", "graph": "the MST workload's graph"}}


def scan_measurement(torch, flush, peak, steps):
    """Exclusive scan of 64 Mi int32 uniform in [0, 1000]: int32 (wrapping,
    8 B per element) and int32 -> int64 (12 B per element) outputs; GB/s
    and fraction of the measured HBM copy bandwidth; end to end through
    exprefixsumNumba with pinned host arrays; CPU: the oracle's restatement
    of exprefixsumNumba (one core)."""
    import ctypes
    import oracle
    from masters_final_b200 import _lib, workloads as W
    from masters_final_b200.utils.scan import exprefixsumNumba
    L = _lib.load()
    n = 64 << 20
    a = W.scan_input(n, seed=3)
    total = int(a.astype(np.int64).sum())
    x = torch.from_numpy(a).cuda()
    tot = torch.empty(1, dtype=torch.int64, device="cuda")
    ws = torch.empty(L.eacb_scan_workspace_size(n), dtype=torch.uint8, device="cuda")
    sh = _lib.stream_handle()
    out = {}
    for name, fn, odt, bpe in (("i32", L.eacb_scan_excl_i32, torch.int32, 8),
                               ("i32_i64", L.eacb_scan_excl_i32_i64, torch.int64, 12)):
        o = torch.empty(n, dtype=odt, device="cuda")

        def step():
            _lib.check(fn(_lib.ptr(x), _lib.ptr(o), n, 0, _lib.ptr(tot), _lib.ptr(ws), ws.numel(),
                          sh), "scan")
        ms = _timed(torch, step, steps, 5, flush)
        gbs = n * bpe / (ms / 1e3) / 1e9
        out[name] = {"ms": ms, "gb_per_s": gbs, "bytes_per_element": bpe,
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak,
                                  "unit": "GB/s", "frac": gbs / peak},
                     "total_exact": int(tot.item()) == total}
        del o
    hin = torch.from_numpy(a).pin_memory()
    hout = torch.empty(n, dtype=torch.int32).pin_memory()
    e_ms = _timed(torch, lambda: exprefixsumNumba(hin, hout), 3, 1, flush)
    out["e2e"] = {"value": n / (e_ms / 1e3), "unit": "elements/s", "ms": e_ms,
                  "h2d_bytes_per_step": 4 * n, "d2h_bytes_per_step": 4 * n,
                  "differences_give_input": bool(np.array_equal(np.diff(hout.numpy()), a[:-1]))}
    # cpu_baseline leg: the oracle, timed
    t0 = time.perf_counter()
    oracle.exprefixsum(a)
    cs = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": n * 8 / cs / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
                           "sample": "64 Mi int32, one run of the oracle's C restatement of "
                                     "exprefixsumNumba"}
    out["config"] = {"workload": "scan_64m", "n": n, "values": "int32 uniform [0, 1000]"}
    return out


# EAC end to end (ensemble -> co-association -> Boruvka MST -> lifetime cut)
EAC_WORKLOADS = {
    # n points, d, mixture components, partitions, k range (np.random.randint,
    # upper bound exclusive), anisotropic, centre range, sigma, seed
    "eac_10k_2d_100p": dict(n=10_000, d=2, comps=6, P=100, k=(50, 101), aniso=False,
                            cr=10.0, sigma=1.0, seed=0),
    "eac_500k_16d_200p": dict(n=500_000, d=16, comps=50, P=200, k=(350, 711), aniso=True,
                              cr=20.0, sigma=1.0, seed=3),
    "eac_2m_8d_100p": dict(n=2_000_000, d=8, comps=200, P=100, k=(700, 1401), aniso=False,
                           cr=50.0, sigma=(0.5, 3.0), seed=5),
}
# many independent datasets in one batched call (EAC.batched.eac_batch): n
# log-uniform in [1000, 50000], d in {2,4,8,16,32}, 3-30 Gaussians with
# sigma U[0.5, 2], centres U[-10, 10]^d, 50 partitions, k range
# [ceil(sqrt(n)/2), ceil(sqrt(n))) per dataset
EAC_BATCHED = dict(instances=512, P=50, seed=0, workers=32)


def eac_run_once(X, cfg, mode, torch):
    """One full EAC pipeline on device-resident data; per-stage CUDA events.
    Returns (stage ms, final labels, the EAC object, the label matrix)."""
    import random
    from masters_final_b200.utils.partition import generate_ensemble_labels
    from masters_final_b200.EAC.eac import EAC
    np.random.seed(cfg["seed"])
    random.seed(cfg["seed"])
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    L, _ = generate_ensemble_labels(X, list(cfg["k"]), cfg["P"], 3, label_mode=mode)
    ev[1].record()
    e = EAC(cfg["n"], sparse=True, condensed=True, n_partitions=cfg["P"])
    e.buildMatrix(L)
    ev[2].record()
    labels = e.finalClustering()
    ev[3].record()
    ev[3].synchronize()
    ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(3)]
    return ms, labels, e, L


def pair_updates(torch, L):
    """Co-association pair updates of a label matrix: sum over partitions and
    clusters of |c| (|c| - 1) / 2 (the reference's inner-loop count)."""
    tot = 0
    for r in L:
        c = torch.bincount(r[r >= 0]).to(torch.int64)
        tot += int((c * (c - 1) // 2).sum().item())
    return tot


def eac_measurements(args):
    """EAC points/s of the BF16 tensor-core and the FP32 pipelines on the
    10k-, 500k- and 2M-point workloads (both pipelines must produce
    identical final partitions), with the reference CPU path beside each
    (the oracle's C restatement, one core: in full at 10k points,
    extrapolated from measured per-stage rates at 500k and 2M); and the
    512-dataset workload batched (BF16) and one dataset at a time (FP32)."""
    import torch
    from masters_final_b200 import workloads as W
    out = {}
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    rates = None
    for name, cfg in EAC_WORKLOADS.items():
        x = W.gaussian_mixture(cfg["n"], cfg["d"], cfg["comps"], seed=cfg["seed"],
                               sigma=cfg["sigma"], center_range=cfg["cr"],
                               anisotropic=cfg["aniso"])
        X = torch.from_numpy(x).cuda()
        small = cfg["n"] <= 50_000
        warm, steps = (3, 5) if small else (1, 1)
        res = {}
        parts = {}
        e = None
        L = None
        # the warm-up run leaves the allocator's cache holding the arrays the
        # timed runs reuse (the stage times are kernels, not cudaMalloc)
        for mode in ("bf16", "cuda"):
            for _ in range(warm):
                e = L = None
                eac_run_once(X, cfg, mode, torch)
            tot = [0.0, 0.0, 0.0]
            for _ in range(steps):
                e = L = None
                flush.fill_(1)
                ms, labels, e, L = eac_run_once(X, cfg, mode, torch)
                tot = [a + b for a, b in zip(tot, ms)]
            total_ms = sum(tot) / steps
            key = "bf16_tc" if mode == "bf16" else "fp32"
            res[key] = {"points_per_s": cfg["n"] / (total_ms / 1000.0), "ms": total_ms,
                        "ms_ensemble": tot[0] / steps, "ms_coassoc": tot[1] / steps,
                        "ms_mst_cut": tot[2] / steps}
            parts[key] = labels
        if not small:
            # the same BF16 run with the built-in launch shapes instead of the
            # autotuner's table
            from masters_final_b200 import _lib
            _lib.clear_tuning()
            try:
                e = L = None
                flush.fill_(1)
                ms_u, _, e, L = eac_run_once(X, cfg, "bf16", torch)
            finally:
                _lib.apply_tuning()
            res["bf16_tc_untuned"] = {"points_per_s": cfg["n"] / (sum(ms_u) / 1000.0),
                                      "ms": sum(ms_u), "ms_ensemble": ms_u[0],
                                      "ms_coassoc": ms_u[1], "ms_mst_cut": ms_u[2],
                                      "tuning": "built-in defaults (table cleared)"}
        res["identical_partitions"] = bool(np.array_equal(parts["bf16_tc"], parts["fp32"]))
        res["nnz"] = int(e.coassoc.nnz)
        res["nnz_discarded"] = int(e.coassoc.nnz_discarded)
        res["n_fclusts"] = int(e.n_fclusts)
        pairs = pair_updates(torch, L)
        res["pair_updates"] = pairs
        res["pair_updates_per_s"] = pairs / (res["bf16_tc"]["ms_coassoc"] / 1e3)
        res["config"] = {k: (list(v) if isinstance(v, tuple) else v) for k, v in cfg.items()}
        if not args.no_cpu_baseline:
            if rates is None:
                res["cpu_baseline"], rates = eac_cpu_full(x, cfg)
            else:
                res["cpu_baseline"] = eac_cpu_extrapolated(x, cfg, rates, pairs, res["nnz"])
        out[name] = res
        del X, e, L
        torch.cuda.empty_cache()
    out["eac_batched_512"] = eac_batched_measurement(torch, args)
    return out


# ------------------------------------------------ EAC reference CPU path --
def _oracle_eac_timed(x, ks, inits, P):
    """The reference EAC pipeline restated on the CPU (oracle, one core):
    per-stage seconds and the work counts."""
    import oracle
    nc, _, nnz, _, secs, pairs = oracle.eac_pipeline(x, ks, inits, P)
    return {"s": secs, "nnz": int(nnz), "pairs": pairs, "n_fclusts": int(nc)}


def eac_cpu_full(x, cfg):
    """The 10k-point workload through the oracle pipeline in full, with the
    same draws as the GPU run; also returns the measured rates that the
    larger workloads are extrapolated from."""
    import random
    from masters_final_b200.utils.partition import draw_ensemble_params
    np.random.seed(cfg["seed"])
    random.seed(cfg["seed"])
    n = x.shape[0]
    ks, inits = draw_ensemble_params(n, list(cfg["k"]), cfg["P"])
    r = _oracle_eac_timed(x, ks, inits, cfg["P"])
    tot = sum(r["s"])
    rates = {"pairs_per_s": r["pairs"] / r["s"][1], "kruskal_entries_per_s": r["nnz"] / r["s"][2]}
    return ({"value": n / tot, "unit": "points/s", "cores": 1, "kind": "port",
             "sample": "the full workload, once: the oracle's C restatement of generateEnsemble "
                       "+ K_Means.fit, EAC_CSR.update_ensemble and sp_sl_lifetime (Kruskal + "
                       "lifetime cut), single-threaded like the reference",
             "stage_s": r["s"], **rates}, rates)


def eac_cpu_extrapolated(x, cfg, rates, pairs, nnz, n_sample=20_000):
    """Reference CPU time of a workload too large to run on the host within
    the bench: the ensemble timed on one partition pair over n_sample
    points (linear in n at fixed k) scaled to n and P; the co-association
    and the Kruskal stage from the pair-update and entry rates the 10k-point
    run measured, applied to this workload's counts (from the GPU run).
    Those rates come from rows of a few hundred entries; the reference's
    sorted-row insertion costs more per pair on longer rows, so the
    estimate is a lower bound of the CPU time."""
    import oracle
    import random
    n = x.shape[0]
    rng = np.random.default_rng(cfg["seed"] + 1)
    xs = np.ascontiguousarray(x[rng.choice(n, n_sample, replace=False)])
    np.random.seed(cfg["seed"])
    random.seed(cfg["seed"])
    ks = [int(np.random.randint(cfg["k"][0], cfg["k"][1])) for _ in range(2)]
    inits = [random.sample(range(n_sample), k) for k in ks]
    t0 = time.perf_counter()
    oracle.ensemble_labels(xs, list(zip(ks, inits)))
    t_ens = (time.perf_counter() - t0) / 2 * (n / n_sample) * cfg["P"]
    t_co = pairs / rates["pairs_per_s"]
    t_fin = nnz / rates["kruskal_entries_per_s"]
    tot = t_ens + t_co + t_fin
    return {"value": n / tot, "unit": "points/s", "cores": 1, "kind": "port",
            "extrapolated": True,
            "sample": "extrapolated: ensemble = 2 partitions on %d sampled points x (n / %d) x "
                      "P; co-association = this workload's %d pair updates at the 10k-point "
                      "run's measured rate; Kruskal = its %d entries at that run's rate"
                      % (n_sample, n_sample, pairs, nnz),
            "stage_s": [t_ens, t_co, t_fin]}


def eac_batched_cpu(xs, ps, P):
    """The 512-dataset workload on the host: a cost-spread sample of
    datasets through the oracle pipeline on one core, and as many datasets
    as host threads through a spawned process pool (one per thread); both
    scaled to all datasets by the instances' relative costs."""
    import multiprocessing as mp
    from masters_final_b200.EAC.batched import instance_cost
    cost = np.array([instance_cost(x.shape[0], x.shape[1], P, max(k))
                     for x, (k, _) in zip(xs, ps)])
    order = np.argsort(cost)
    N = float(sum(x.shape[0] for x in xs))
    # samples from the lower two-thirds of the cost range keep this leg to
    # tens of seconds; the scaling by relative cost covers the rest
    hi = max(1, int(0.65 * (len(xs) - 1)))
    one = order[np.linspace(int(0.2 * hi), hi, 4).round().astype(int)]
    import oracle
    t1 = sum(oracle.eac_pipeline_seconds((xs[i], ps[i][0], ps[i][1], P)) for i in one)
    est1 = t1 * cost.sum() / cost[one].sum()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    cores = max(1, min(cores or 1, 64))
    many = order[np.linspace(int(0.15 * hi), hi, cores).round().astype(int)]
    with mp.get_context("spawn").Pool(cores) as pool:
        pool.map(oracle.eac_pipeline_seconds,
                 [(xs[one[0]], ps[one[0]][0], ps[one[0]][1], P)] * cores)
        t0 = time.perf_counter()
        pool.map(oracle.eac_pipeline_seconds, [(xs[i], ps[i][0], ps[i][1], P) for i in many],
                 chunksize=1)
        tw = time.perf_counter() - t0
    estn = tw * cost.sum() / cost[many].sum()
    return {"value": N / est1, "unit": "points/s", "cores": 1, "kind": "port",
            "extrapolated": True,
            "sample": "4 datasets from the lower two-thirds of the cost range through the oracle "
                      "pipeline on one core (%.1f s), scaled to all %d by relative cost "
                      "(EAC.batched.instance_cost)" % (t1, len(xs)),
            "host": {"value": N / estn, "unit": "points/s", "cores": cores,
                     "sample": "%d datasets on %d spawned processes at once (%.1f s wall), "
                               "scaled to all %d by relative cost" % (cores, cores, tw, len(xs))}}


def eac_batched_sharded_measurement(torch, dist, world):
    """The batched workload split across the ranks (instances balanced by
    cost, one exchange of results at the end): Σn / max-over-ranks time of
    one eac_batch_distributed call, after one warm-up call."""
    from masters_final_b200 import workloads as W
    from masters_final_b200.EAC.batched import eac_batch_distributed
    cfg = EAC_BATCHED
    xs = W.batched_instances(cfg["instances"], seed=cfg["seed"])
    N = int(sum(x.shape[0] for x in xs))
    eac_batch_distributed(xs, cfg["P"], n_workers=cfg["workers"])
    dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = eac_batch_distributed(xs, cfg["P"], n_workers=cfg["workers"])
    torch.cuda.synchronize()
    t = torch.tensor([time.perf_counter() - t0], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dt = float(t.item())
    return {"points_per_s": N / dt, "s": dt, "sum_n": N, "instances": len(xs),
            "n_gpus": world, "scaling": "strong", "failed": int(sum(r.status != 0 for r in out)),
            "timing": "host wall clock around the call, max over ranks (the call ends with "
                      "an exchange of results)",
            "config": {**cfg, "label_mode": "bf16"}}


def eac_batched_measurement(torch, args):
    """Batched EAC points/s (sum of n over all datasets / wall time of one
    eac_batch call, BF16 labels, data on the device), after one warm-up
    call; beside it the same datasets run one at a time through the
    single-instance pipeline with the FP32 labeler, whose final partitions
    must be identical; and the reference CPU path."""
    import random
    from masters_final_b200 import workloads as W
    from masters_final_b200.EAC.batched import eac_batch, draw_instance_params, k_range_rule1
    from masters_final_b200.EAC.eac import eac_pipeline
    cfg = EAC_BATCHED
    xs = W.batched_instances(cfg["instances"], seed=cfg["seed"])
    ps = [draw_instance_params(x.shape[0], k_range_rule1(x.shape[0]), cfg["P"], i)
          for i, x in enumerate(xs)]
    from masters_final_b200 import _lib
    Xd = [torch.from_numpy(x).cuda() for x in xs]
    N = int(sum(x.shape[0] for x in xs))
    workers = int(_lib.tuned("batched_workers", cfg["workers"]))
    eac_batch(Xd, params=ps, n_workers=workers, return_device=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = eac_batch(Xd, params=ps, n_workers=workers, return_device=True)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    # untuned: the built-in launch shapes and the default worker count
    _lib.clear_tuning()
    try:
        eac_batch(Xd, params=ps, return_device=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eac_batch(Xd, params=ps, return_device=True)
        torch.cuda.synchronize()
        du = time.perf_counter() - t0
    finally:
        _lib.apply_tuning()
    st = np.array([a.ms_stages for a in r])
    out = {"points_per_s": N / dt, "s": dt, "sum_n": N, "instances": len(xs),
           "nnz_total": int(sum(a.nnz for a in r)),
           "nnz_discarded_total": int(sum(a.nnz_discarded for a in r)),
           "failed": int(sum(a.status != 0 for a in r)),
           "worker_ms_sums": {"ensemble": float(st[:, 0].sum()), "coassoc": float(st[:, 1].sum()),
                              "final": float(st[:, 2].sum())},
           "untuned": {"points_per_s": N / du, "s": du,
                       "tuning": "built-in defaults (table cleared, default worker count)"},
           "config": {**cfg, "workers": workers, "n_range": [1000, 50000],
                      "d": [2, 4, 8, 16, 32], "gaussians": [3, 30], "sigma": [0.5, 2.0],
                      "label_mode": "bf16"}}
    # the plain single-instance pipeline: FP32 labeler, one dataset at a time
    def single(i):
        np.random.seed(i)
        random.seed(i)
        return eac_pipeline(Xd[i], cfg["P"], k_range_rule1(xs[i].shape[0]), label_mode="cuda")
    single(0)
    torch.cuda.synchronize()
    same = True
    t0 = time.perf_counter()
    for i in range(len(xs)):
        nf, lab, _ = single(i)
        rb = r[i]
        if rb.labels_valid:
            same = same and nf == rb.n_fclusts and np.array_equal(lab, rb.labels.cpu().numpy())
        else:
            same = same and nf <= 1
    torch.cuda.synchronize()
    ds = time.perf_counter() - t0
    out["single_instance_fp32"] = {"points_per_s": N / ds, "s": ds, "identical_partitions": same,
                                   "timing": "host wall clock around 512 sequential "
                                             "eac_pipeline calls (label_mode cuda)"}
    out["batched_over_single_fp32"] = (N / dt) / (N / ds)
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = eac_batched_cpu(xs, ps, cfg["P"])
    return out


# ------------------------------------------------- profiling cases --------
def case_label_tc_100k():
    """K-Means ensemble on the tensor-core labeler: 100,000 16-D points from
    50 anisotropic Gaussians (the 500k workload's mixture), 2 partitions, k
    in [350, 711), 3 Lloyd iterations."""
    import torch
    from masters_final_b200 import workloads as W
    from masters_final_b200.cluster.KMeans import kmeans_ensemble
    x = W.gaussian_mixture(100_000, 16, 50, seed=3, center_range=20.0, anisotropic=True)
    rng = np.random.default_rng(4)
    ks = [int(k) for k in rng.integers(350, 711, 2)]
    inits = [rng.choice(x.shape[0], k, replace=False).tolist() for k in ks]
    X = torch.from_numpy(x).cuda()
    for _ in range(2):
        out = kmeans_ensemble(X, ks, inits, max_iter=3, label_mode="bf16")
    torch.cuda.synchronize()
    return {"ks": ks, "iters": out[3].tolist()}


def case_ensemble_500k_20p():
    """K-Means ensemble of the 500,000-point workload's data (16-D, 50
    anisotropic Gaussians) with 20 of its 200 partitions (k in [350, 711),
    3 Lloyd iterations, BF16 labeler): every kernel of the ensemble stage."""
    import random
    import torch
    from masters_final_b200 import workloads as W
    from masters_final_b200.utils.partition import generate_ensemble_labels
    x = W.gaussian_mixture(500_000, 16, 50, seed=3, center_range=20.0, anisotropic=True)
    X = torch.from_numpy(x).cuda()
    np.random.seed(3)
    random.seed(3)
    for _ in range(2):
        L, ks = generate_ensemble_labels(X, [350, 711], 20, 3, label_mode="bf16")
    torch.cuda.synchronize()
    return {"partitions": len(ks)}


def case_batched_64():
    """Batched EAC of every eighth of the 512 datasets (64 instances, n
    from 1,000 to 50,000, 50 partitions, BF16 labels), two calls."""
    import torch
    from masters_final_b200 import workloads as W
    from masters_final_b200.EAC.batched import draw_instance_params, eac_batch, k_range_rule1
    xs = W.batched_instances(EAC_BATCHED["instances"], seed=EAC_BATCHED["seed"])
    ps = [draw_instance_params(x.shape[0], k_range_rule1(x.shape[0]), EAC_BATCHED["P"], i)
          for i, x in enumerate(xs)][::8]
    Xd = [torch.from_numpy(x).cuda() for x in xs[::8]]
    for _ in range(2):
        r = eac_batch(Xd, params=ps, return_device=True)
    torch.cuda.synchronize()
    return {"instances": len(Xd), "sum_n": int(sum(x.shape[0] for x in Xd)),
            "failed": int(sum(a.status != 0 for a in r))}


def case_mst_knn16_1M():
    """Three Boruvka MST calls on the 16-NN graph of 1,000,000 points."""
    import torch
    from masters_final_b200 import workloads as W
    from masters_final_b200.graph.mst import boruvka_minho_gpu
    indptr, dest, w = W.knn_graph(N_VERTICES, k=KNN, seed=SEED)
    d = [torch.from_numpy(a).cuda() for a in (dest, w, indptr[:-1].astype(np.int32),
                                               np.diff(indptr).astype(np.int32))]
    for _ in range(3):
        _, n = boruvka_minho_gpu(*d, returnDevAry=True)
    torch.cuda.synchronize()
    return {"n_mst": n}


def case_coassoc300k():
    """Co-association count and fill of 300,000 16-D points from 50
    anisotropic Gaussians (centres in [-20, 20]^16), 100 K-Means partitions
    with k in [210, 427) (BF16 labels), linear capacity, factor 3."""
    import random
    import torch
    from masters_final_b200 import workloads as W
    from masters_final_b200.EAC.sparse import CoassocBuilder, EAC_CSR
    from masters_final_b200.utils.partition import generate_ensemble_labels
    x = W.gaussian_mixture(300_000, 16, 50, seed=3, center_range=20.0, anisotropic=True)
    np.random.seed(3)
    random.seed(3)
    L, _ = generate_ensemble_labels(torch.from_numpy(x).cuda(), [210, 427], 100, 3,
                                    label_mode="bf16")
    b = CoassocBuilder(L, x.shape[0])
    c = EAC_CSR(x.shape[0], max_assocs=int(b.max_cluster * 3), condensed=True,
                max_assocs_type="linear")
    c.update_ensemble(None, builder=b)
    torch.cuda.synchronize()
    return {"nnz": int(c.nnz)}


def case_final_phase_synthetic():
    """EAC final clustering of a synthetic condensed matrix: 100,000 rows,
    row i holding min(5000, n-1-i) columns spread over (i, n), uint8 weights
    101 - floor(100 u^0.25), max_dist 100."""
    import torch
    from masters_final_b200.EAC.eac import sp_sl_lifetime_csr
    n, m = 100_000, 5000
    rng = np.random.default_rng(6)
    deg = np.minimum(m, n - 1 - np.arange(n)).astype(np.int64)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(deg, out=indptr[1:])
    rows = np.repeat(np.arange(n), deg)
    span = (n - 1 - rows).astype(np.float64)
    pos = np.arange(indptr[-1]) - indptr[rows]
    cols = (rows + 1 + np.floor(pos * span / np.maximum(deg[rows], 1))).astype(np.int32)
    w = (101 - np.floor(100 * rng.random(pos.size) ** 0.25)).astype(np.uint8)
    d = [torch.from_numpy(a).cuda() for a in (indptr, cols, w)]
    nc, _ = sp_sl_lifetime_csr(d[0], d[1], d[2], n, 100, returnDevAry=True)
    torch.cuda.synchronize()
    return {"entries": int(indptr[-1]), "n_fclusts": int(nc)}


CASES = {"label_tc_100k": case_label_tc_100k, "ensemble_500k_20p": case_ensemble_500k_20p,
         "batched_64": case_batched_64, "mst_knn16_1M": case_mst_knn16_1M,
         "coassoc300k": case_coassoc300k, "final_phase_synthetic": case_final_phase_synthetic}


def main():
    args = parse()
    if args.case:
        print(json.dumps({"case": args.case, **CASES[args.case]()}), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
