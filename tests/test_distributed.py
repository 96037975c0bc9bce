"""Batch sharding over ranks (CPU): the longest-processing-time assignment,
and the SUM all-reduce that assembles energies and gradients, run as two gloo
ranks on 127.0.0.1 with a host-side stand-in for the per-rank GPU evaluation."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from kettle_b200 import distributed as D


def test_shards_cover_every_item_once_and_balance():
    rng = np.random.default_rng(0)
    q = rng.integers(10, 23, size=500)
    g = rng.integers(50, 700, size=500)
    costs = [D.item_cost(a, b) for a, b in zip(q, g)]
    for world in (1, 2, 3, 8):
        shards = D.shard_items(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(500))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(costs)
        assert D.shard_items(costs, world) == shards  # deterministic


def test_gather_without_processes():
    e, g = D.gather([3.0, 1.0], [2, 0], 3, np.arange(4.0))
    assert list(e) == [1.0, 0.0, 3.0]
    assert list(g) == [0.0, 1.0, 2.0, 3.0]


def _fake_rank_result(shard, param_ranges, n_params):
    """What a rank's kt_batch returns, with energy_i = 10 i and, for every
    parameter p its items bind, dE/dp = p + 0.5 per binding item."""
    e = np.array([10.0 * i for i in shard])
    g = np.zeros(n_params)
    for i in shard:
        lo, hi = param_ranges[i]
        g[lo:hi] += np.arange(lo, hi) + 0.5
    return e, g


def _worker(rank, world, port, costs, param_ranges, n_params, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shard = D.shard_items(costs, world)[rank]
        e, g = _fake_rank_result(shard, param_ranges, n_params)
        e_all, g_all = D.gather(e, shard, len(costs), g, dist)
        out_q.put((rank, e_all.tolist(), g_all.tolist()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2])
def test_gather_over_gloo_ranks(world):
    rng = np.random.default_rng(1)
    n_items = 37
    sizes = rng.integers(1, 6, size=n_items)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    param_ranges = [(int(a), int(a + b)) for a, b in zip(starts, sizes)]
    param_ranges[5] = param_ranges[4]      # two items sharing one parameter range
    n_params = int(sizes.sum())
    costs = [D.item_cost(q, gcount) for q, gcount in zip(rng.integers(10, 23, n_items), rng.integers(10, 300, n_items))]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, costs, param_ranges, n_params, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want_e, want_g = _fake_rank_result(list(range(n_items)), param_ranges, n_params)
    for _, e, g in results:
        assert np.array_equal(np.array(e), want_e)
        assert np.allclose(np.array(g), want_g, rtol=0, atol=1e-12)


def test_string_and_parameter_shards_cover_once():
    rng = np.random.default_rng(3)
    x = rng.integers(0, 8, size=200)  # many strings per X mask
    for world in (1, 2, 3):
        shards = D.shard_strings(x, world)
        assert sorted(i for s in shards for i in s) == list(range(200))
        for s in shards:  # a mask group never straddles two ranks
            for t in shards:
                if s is not t:
                    assert not set(x[s]) & set(x[t])
        ps = D.shard_params(17, world)
        assert sorted(i for s in ps for i in s) == list(range(17))


def _fake_terms(strings, coeffs):
    return (strings["x"] + 0.5) * np.exp(0.25j * strings["z"])


def _fake_energy(p):
    return float(np.sum(np.sin(p) * np.arange(1, p.size + 1)))


def _worker_units(rank, world, port, strings, coeffs, params, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        terms, total = D.sharded_expectation(_fake_terms, strings, coeffs, rank, world, dist)
        grad = D.sharded_parameter_shift(_fake_energy, params, rank, world, dist)
        out_q.put((rank, terms.tolist(), total, grad.tolist()))
    finally:
        dist.destroy_process_group()


def test_sharded_strings_and_shifts_over_gloo_ranks():
    """Two gloo ranks: every rank gets every string's term, the same total
    (bit for bit) and the same parameter-shift gradient as one process."""
    from kettle_b200 import capi
    rng = np.random.default_rng(4)
    strings = np.zeros(41, dtype=capi.PAULI_DTYPE)
    strings["x"] = rng.integers(0, 6, size=41)
    strings["z"] = rng.integers(0, 64, size=41)
    coeffs = rng.normal(size=41) + 1j * rng.normal(size=41)
    params = rng.uniform(-3, 3, size=13)
    want_terms, want_total = D.sharded_expectation(_fake_terms, strings, coeffs, 0, 1)
    want_grad = D.sharded_parameter_shift(_fake_energy, params, 0, 1)
    assert np.abs(want_grad - np.cos(params) * np.arange(1, 14)).max() < 1e-12
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_units, args=(r, world, port, strings, coeffs, params, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, terms, total, grad in got:
        assert np.array_equal(np.array(terms), want_terms), rank
        assert total == want_total, rank
        assert np.array_equal(np.array(grad), want_grad), rank
