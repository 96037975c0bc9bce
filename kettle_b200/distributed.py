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


# ---------------------------------------------------------------------------
# Pauli-string lists and parameter-shift shifts, the other independent units.
# Every rank holds the same state (the statevector path runs as replicas),
# evaluates its share of the units, and one SUM all-reduce of a vector with
# one slot per unit — each slot written by exactly one rank — assembles the
# values on every rank; totals are then formed in unit order, so every rank
# gets the same bits.

def shard_strings(x_masks, world: int) -> list[list[int]]:
    """String indices per rank.  Strings with one X/Y mask share one read of
    the state (k_pauli's slot), so whole mask groups are assigned, by the
    longest-processing-time rule on their cost (one state read per 16
    strings of the group)."""
    groups: dict[int, list[int]] = {}
    for i, x in enumerate(x_masks):
        groups.setdefault(int(x), []).append(i)
    keys = list(groups)
    costs = [float((len(groups[k]) + 15) // 16) for k in keys]
    out: list[list[int]] = [[] for _ in range(world)]
    for r, sel in enumerate(shard_items(costs, world)):
        for g in sel:
            out[r].extend(groups[keys[g]])
    return [sorted(s) for s in out]


def shard_params(n_params: int, world: int) -> list[list[int]]:
    """Parameter indices per rank for the parameter-shift rule (two shifted
    energies of equal cost per parameter): round robin."""
    if world < 1:
        raise ValueError("world must be >= 1")
    return [list(range(r, n_params, world)) for r in range(world)]


def gather_units(values_local, indices, n: int, dist=None, group=None, device=None) -> np.ndarray:
    """The full vector of n unit values on every rank: `values_local[k]`
    (real or complex) belongs to unit `indices[k]`."""
    vals = np.asarray(values_local)
    cplx = np.iscomplexobj(vals)
    full = np.zeros(n, dtype=np.complex128 if cplx else np.float64)
    full[np.asarray(indices, dtype=np.int64)] = vals
    if dist is None:
        return full
    import torch
    flat = np.concatenate([full.real, full.imag]) if cplx else full
    t = torch.from_numpy(np.ascontiguousarray(flat)).to(device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    out = t.cpu().numpy()
    return out[:n] + 1j * out[n:] if cplx else out.copy()


def sharded_expectation(evaluate_terms, strings, coeffs, rank: int, world: int, dist=None, group=None,
                        device=None):
    """<H> = sum_k c_k <P_k> of this rank's replica with the strings sharded:
    `evaluate_terms(strings_subset, coeffs_subset)` returns this rank's terms
    (complex, the strings' phases included; e.g. capi.Statevector.expect's
    first result).  Returns (all terms, total), the same on every rank."""
    strings = np.ascontiguousarray(strings, dtype=capi.PAULI_DTYPE)
    c = np.ones(strings.size, dtype=np.complex128) if coeffs is None else np.asarray(coeffs, dtype=np.complex128)
    mine = shard_strings(strings["x"], world)[rank]
    local = evaluate_terms(strings[mine], c[mine]) if mine else np.zeros(0, dtype=np.complex128)
    terms = gather_units(np.asarray(local, dtype=np.complex128), mine, strings.size, dist, group, device)
    return terms, complex(np.sum(c * terms))


def sharded_parameter_shift(energy, params, rank: int, world: int, dist=None, group=None, device=None,
                            shift: float = np.pi / 2) -> np.ndarray:
    """dE/dθ_p = (E(θ + s e_p) − E(θ − s e_p)) / 2 (the rule for RX/RY/RZ
    slots, s = π/2) with the parameters sharded over ranks; `energy(θ)` runs
    on this rank's GPU.  The full gradient on every rank."""
    p = np.asarray(params, dtype=np.float64)
    mine = shard_params(p.size, world)[rank]
    local = []
    for k in mine:
        up, dn = p.copy(), p.copy()
        up[k] += shift
        dn[k] -= shift
        local.append(0.5 * (float(energy(up)) - float(energy(dn))))
    return gather_units(np.asarray(local, dtype=np.float64), mine, p.size, dist, group, device)
