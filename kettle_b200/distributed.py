"""Batches over several GPUs: one process per GPU, items sharded by cost.

The batch configuration's items are independent, so a multi-GPU run needs no
exchange while it computes: every rank evaluates its own shard with one
kt_batch (a CUDA graph on its GPU), and one collective at the end — a SUM
all-reduce of the energy and gradient vectors, kilobytes long — assembles the
result on every rank (NCCL over NVLink on GPUs; gloo in the CPU tests).  The
shards are disjoint, so the sum is a gather for the energies; for gradients it
is also the batch's own rule (grads[p] sums over every item that binds p).

Sharding is the longest-processing-time rule on the item cost 2^q * (gates+1):
items in decreasing cost, each to the rank with the least work so far (ties to
the lower rank), which keeps the slowest rank within one item of the mean.
"""
from __future__ import annotations

import heapq

import numpy as np

from . import capi


def item_cost(n_qubits: int, n_gates: int) -> float:
    return float(2 ** int(n_qubits)) * float(int(n_gates) + 1)


def shard_items(costs, world: int) -> list[list[int]]:
    """Indices of the items each rank evaluates (each list in increasing order)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in shards]


def gather(energies_local, shard, n_items: int, grads_local, dist=None, group=None, device=None):
    """Assemble the full energy (n_items) and gradient vectors on every rank.

    `energies_local[k]` belongs to item `shard[k]`; `grads_local` is this rank's
    full-length gradient vector (zero where its items bind no parameter) or
    None.  With `dist` None (one process) the inputs are only reassembled."""
    e = np.zeros(n_items, dtype=np.float64)
    e[np.asarray(shard, dtype=np.int64)] = np.asarray(energies_local, dtype=np.float64)
    g = None if grads_local is None else np.asarray(grads_local, dtype=np.float64).copy()
    if dist is None:
        return e, g
    import torch
    dev = device if device is not None else "cpu"
    parts = [e] if g is None else [e, g]
    flat = torch.from_numpy(np.concatenate(parts)).to(dev)
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    out = flat.cpu().numpy()
    e = out[:n_items].copy()
    g = None if g is None else out[n_items:].copy()
    return e, g


class ShardedBatch:
    """This rank's share of a batch: a kt_batch over its items (the flat gate,
    parameter and Pauli arrays are the whole batch's, so parameter indices
    stay global), and `evaluate` returns the whole batch's result."""

    def __init__(self, items, gates, strings, coeffs, n_params: int, rank: int, world: int, dtype: int = capi.KT_C128,
                 with_grad: bool = True, dist=None, group=None, device=None):
        items = np.ascontiguousarray(items, dtype=capi.BATCH_ITEM_DTYPE)
        costs = [item_cost(it["n_qubits"], it["n_gates"]) for it in items]
        self.shards = shard_items(costs, world)
        self.shard = self.shards[rank]
        self.n_items = items.size
        self.n_params = int(n_params)
        self.with_grad = with_grad
        self.dist, self.group, self.device = dist, group, device
        self.local = None
        if self.shard:
            self.local = capi.Batch(items[self.shard], gates, strings, coeffs, n_params, dtype=dtype,
                                    with_grad=with_grad)

    def evaluate_local(self, params):
        """This rank's energies (in shard order) and full-length gradients."""
        if self.local is None:
            return np.zeros(0), (np.zeros(self.n_params) if self.with_grad else None)
        return self.local.evaluate(params)

    def evaluate(self, params):
        e, g = self.evaluate_local(params)
        return gather(e, self.shard, self.n_items, g, self.dist, self.group, self.device)

    def close(self):
        if self.local is not None:
            self.local.close()
            self.local = None
