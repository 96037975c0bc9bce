"""The sharded batch (kettle_b200.distributed.ShardedBatch) on the engine.

Two ranks run as two processes on one GPU, joined by a gloo process group on
127.0.0.1: the only collective is the host-side SUM all-reduce that
assembles the energies and gradients, so neither rank's kernels wait on the
other's.  Each rank builds a kt_batch over its cost-balanced share of 24
hardware-efficient-ansatz instances (8..15 qubits: shared-memory and HBM
items, compiled classes included) and evaluates it twice with different
parameters (the second a graph replay).  Every rank must hold the whole
batch's energies and gradients, equal to one unsharded kt_batch over the
same instances (1e-12: each item's work is the same kernels on the same
data whichever companions it has; gradient slots are written by exactly one
rank)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from kettle_b200 import capi
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu

N_ITEMS = 24


def _workload():
    circuits, params = W.hea_batch(N_ITEMS, seed=77, qubits=(8, 15), layers=(2, 4), n_strings=12)
    rng = np.random.default_rng(78)
    return circuits, params, rng.uniform(-np.pi, np.pi, params.size)


def _rank(rank, world, port, out_q):
    import datetime

    import torch
    import torch.distributed as dist

    from kettle_b200 import distributed as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    sb = None
    try:
        circuits, p1, p2 = _workload()
        items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
        sb = D.ShardedBatch(items, gates, strings, coeffs, n_params, rank, world, dist=dist)
        e1, g1 = sb.evaluate(p1)
        e2, g2 = sb.evaluate(p2)
        out_q.put((rank, list(sb.shard), e1, g1, e2, g2))
    finally:
        if sb is not None:
            sb.close()
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_batch_over_two_ranks_equals_unsharded(engine):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        results = [q.get(timeout=600) for _ in range(world)]
    finally:
        for p in procs:
            p.join(timeout=120)
    assert [p.exitcode for p in procs] == [0] * world

    circuits, p1, p2 = _workload()
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    b = capi.Batch(items, gates, strings, coeffs, n_params)
    want1 = b.evaluate(p1)
    want2 = b.evaluate(p2)
    b.close()

    shards = sorted(i for _, shard, *_ in results for i in shard)
    assert shards == list(range(N_ITEMS))  # every item on exactly one rank
    assert all(len(shard) > 0 for _, shard, *_ in results)
    for _, _, e1, g1, e2, g2 in results:
        for (e, g), (we, wg) in (((e1, g1), want1), ((e2, g2), want2)):
            assert e.shape == we.shape and g.shape == wg.shape
            assert np.abs(e - we).max() < 1e-12
            assert np.abs(g - wg).max() < 1e-12
    assert np.abs(want1[1] - want2[1]).max() > 1e-3  # the second parameters did change the result
