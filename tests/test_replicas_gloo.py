"""Multi-process replica plumbing on CPU (gloo, world size 2).

The multi-GPU path is replicas only: each rank runs its own ion or requests,
and only scalar timings are reduced. These tests run the same host code as
``bench.py --gpus N`` on two gloo ranks: max and sum reductions, the barrier,
rank-dependent replica seeds (different ions per rank), and the cost-balanced
sharding of the uneven batch.
"""
import os
import socket

import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from atomx_b200 import replicas
    from atomx_b200 import workloads as W
    r, w, _ = replicas.init("gloo", timeout_s=60)
    replicas.barrier(w)
    mx = replicas.reduce_max(10.0 + r, w)
    sm = replicas.reduce_sum(1.0 + r, w)
    spec = W.ytterbium_scaleup(seed=replicas.replica_seed(2026, r))
    replicas.barrier(w)
    replicas.finalize(w)
    out.put((r, mx, sm, spec.seed))


def test_two_gloo_ranks_reduce_and_seed_replicas():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] == 11.0 and r[2] == 3.0 for r in res)   # max over ranks, sum over ranks
    assert res[0][3] != res[1][3]                              # each rank its own seeded ion


def test_shard_balances_the_uneven_batch():
    from atomx_b200 import replicas
    from atomx_b200 import workloads as W
    specs = W.uneven_batch()
    cost = [s.ns * sum(c for _, c in s.shells) ** 2 for s in specs]
    for world in (1, 2, 4, 8):
        parts = replicas.shard(cost, world)
        assert sorted(i for p in parts for i in p) == list(range(len(specs)))
        loads = [sum(cost[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(cost)
