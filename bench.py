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
     "per round: 8 B per edge word read + 8 B per surviving word written + 8 B per original "
     "vertex (label read and written) + 24 B per supervertex (selection slot, successor, "
     "new id)"),
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
        if world == 1 and not args.no_eac:
            line["eac"] = eac_measurements(args)
        if sharded is not None:
            line["eac_batched_sharded"] = sharded
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


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
    """One full EAC pipeline on device-resident data; per-stage CUDA events."""
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
    return ms, labels, e


def eac_measurements(args):
    """EAC points/s of the BF16 tensor-core and the FP32 pipelines on the
    10k-point (reference CPU-runnable) and 500k-point workloads; both
    pipelines must produce identical final partitions."""
    import torch
    from masters_final_b200 import workloads as W
    out = {}
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
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
        def release():
            # large workloads: the previous matrix goes before the next one is
            # built (small ones keep the allocator's cache, as a user would)
            if not small:
                torch.cuda.empty_cache()
        for mode in ("bf16", "cuda"):
            for _ in range(warm):
                e = None
                release()
                eac_run_once(X, cfg, mode, torch)
            tot = [0.0, 0.0, 0.0]
            for _ in range(steps):
                e = None
                release()
                flush.fill_(1)
                ms, labels, e = eac_run_once(X, cfg, mode, torch)
                tot = [a + b for a, b in zip(tot, ms)]
            total_ms = sum(tot) / steps
            key = "bf16_tc" if mode == "bf16" else "fp32"
            res[key] = {"points_per_s": cfg["n"] / (total_ms / 1000.0), "ms": total_ms,
                        "ms_ensemble": tot[0] / steps, "ms_coassoc": tot[1] / steps,
                        "ms_mst_cut": tot[2] / steps}
            parts[key] = labels
        res["identical_partitions"] = bool(np.array_equal(parts["bf16_tc"], parts["fp32"]))
        res["nnz"] = int(e.coassoc.nnz)
        res["nnz_discarded"] = int(e.coassoc.nnz_discarded)
        res["n_fclusts"] = int(e.n_fclusts)
        res["config"] = {k: (list(v) if isinstance(v, tuple) else v) for k, v in cfg.items()}
        out[name] = res
        del X, e
        torch.cuda.empty_cache()
    out["eac_batched_512"] = eac_batched_measurement(torch)
    return out


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


def eac_batched_measurement(torch):
    """Batched EAC points/s (sum of n over all datasets / wall time of one
    eac_batch call, data on the device), after one warm-up call."""
    from masters_final_b200 import workloads as W
    from masters_final_b200.EAC.batched import eac_batch, draw_instance_params, k_range_rule1
    cfg = EAC_BATCHED
    xs = W.batched_instances(cfg["instances"], seed=cfg["seed"])
    ps = [draw_instance_params(x.shape[0], k_range_rule1(x.shape[0]), cfg["P"], i)
          for i, x in enumerate(xs)]
    Xd = [torch.from_numpy(x).cuda() for x in xs]
    N = int(sum(x.shape[0] for x in xs))
    eac_batch(Xd, params=ps, n_workers=cfg["workers"], return_device=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = eac_batch(Xd, params=ps, n_workers=cfg["workers"], return_device=True)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    st = np.array([a.ms_stages for a in r])
    return {"points_per_s": N / dt, "s": dt, "sum_n": N, "instances": len(xs),
            "nnz_total": int(sum(a.nnz for a in r)),
            "nnz_discarded_total": int(sum(a.nnz_discarded for a in r)),
            "failed": int(sum(a.status != 0 for a in r)),
            "worker_ms_sums": {"ensemble": float(st[:, 0].sum()), "coassoc": float(st[:, 1].sum()),
                               "final": float(st[:, 2].sum())},
            "config": {**cfg, "n_range": [1000, 50000], "d": [2, 4, 8, 16, 32],
                       "gaussians": [3, 30], "sigma": [0.5, 2.0], "label_mode": "bf16"}}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
