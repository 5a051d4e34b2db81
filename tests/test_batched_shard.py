"""Host logic of the multi-GPU batched EAC (instances sharded across ranks,
one exchange of results at the end), on CPU with gloo and a stand-in for
the per-rank GPU call."""
import os
import socket

import numpy as np
import pytest


def _fake_runner(xs, n_partitions, params, **kw):
    """Deterministic stand-in for eac_batch: encodes each instance's data and
    host draws into its result."""
    from masters_final_b200.EAC.batched import BatchResult
    out = []
    for x, (ks, inits) in zip(xs, params):
        lab = np.full(x.shape[0], int(abs(float(x[0, 0])) * 1000) % 97, dtype=np.int32)
        out.append(BatchResult(lab, len(ks), int(sum(ks)), int(sum(map(sum, inits))) % 1000, 1, 0))
    return out


def _instances(m=9, seed=4):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((int(rng.integers(200, 3000)), int(rng.choice([2, 8]))))
            .astype(np.float32) for _ in range(m)]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from masters_final_b200.EAC.batched import eac_batch_distributed
        out = eac_batch_distributed(_instances(), n_partitions=6, runner=_fake_runner)
        q.put((rank, [(int(r.labels[0]), r.n_fclusts, r.nnz, r.nnz_discarded) for r in out]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_instances_balanced():
    from masters_final_b200.EAC.batched import shard_instances
    costs = [9, 7, 6, 5, 4, 3, 2, 2, 1]
    parts = shard_instances(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)


def test_distributed_batch_matches_single_process():
    import torch.multiprocessing as mp
    from masters_final_b200.EAC.batched import draw_instance_params, k_range_rule1
    xs = _instances()
    expect = []
    for i, x in enumerate(xs):
        ks, inits = draw_instance_params(x.shape[0], k_range_rule1(x.shape[0]), 6, i)
        r = _fake_runner([x], 6, [(ks, inits)])[0]
        expect.append((int(r.labels[0]), r.n_fclusts, r.nnz, r.nnz_discarded))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0] == expect
    assert got[1] == expect
