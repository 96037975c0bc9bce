"""Autotuner for the fused-block launch shape (no reference counterpart).

The fused kernels take three knobs (kt_tuning_set): the tile size
(`fused_tile_bits`, 9..13 qubits for complex128, one more for complex64), the
number of gates a block may take (`fused_max_ops`, the fusion depth), and the
register budget (`fused_ctas_per_sm`: 2 CTAs per SM at <= 128 registers, or 1
with the compiler's natural allocation).  `autotune` times `kt_sv_apply` on a
seeded random circuit of the requested size over a grid of candidates on the
current GPU, keeps the fastest, sets it, and caches it per (GPU name, dtype,
qubit count) in a JSON file, so later processes reuse it with `load`.

Every candidate computes the same amplitudes up to FP64 rounding (the knobs
only regroup gates into blocks); the tests check that.
"""
from __future__ import annotations

import itertools
import json
import os
import pathlib
import time
from typing import Callable, Iterable

from . import capi

KNOBS = ("fused_tile_bits", "fused_max_ops", "fused_ctas_per_sm")
DEFAULT_GRID = {
    "fused_tile_bits": (10, 11, 12, 13),
    "fused_max_ops": (64, 128, 256),
    "fused_ctas_per_sm": (1, 2),
}


def cache_path() -> pathlib.Path:
    """KT_TUNING_CACHE, else ~/.cache/kettle_b200/tuning.json."""
    env = os.environ.get("KT_TUNING_CACHE")
    if env:
        return pathlib.Path(env)
    return pathlib.Path.home() / ".cache" / "kettle_b200" / "tuning.json"


def _key(device: str, dtype: int, n_qubits: int) -> str:
    return f"{device}|{'c128' if dtype == capi.KT_C128 else 'c64'}|{n_qubits}"


def candidates(grid: dict | None = None) -> list[dict]:
    """All knob combinations of `grid` (defaults to DEFAULT_GRID), in a fixed order."""
    g = dict(DEFAULT_GRID)
    if grid:
        g.update(grid)
    return [dict(zip(KNOBS, combo)) for combo in itertools.product(*(g[k] for k in KNOBS))]


def current() -> dict:
    return {k: capi.tuning_get(k) for k in KNOBS}


def set_knobs(knobs: dict) -> None:
    for k, v in knobs.items():
        capi.tuning_set(k, int(v))


def search(timer: Callable[[dict], float], cands: Iterable[dict]) -> tuple[dict, list]:
    """Time every candidate with `timer(knobs) -> seconds`; return (best, table).
    Ties keep the earlier candidate."""
    table = []
    best, best_t = None, float("inf")
    for c in cands:
        t = float(timer(c))
        table.append({**c, "seconds": t})
        if t < best_t:
            best, best_t = c, t
    if best is None:
        raise ValueError("no candidates")
    return best, table


def _device_name() -> str:
    import torch
    return torch.cuda.get_device_name()


def gpu_timer(n_qubits: int, dtype: int = capi.KT_C128, layers: int = 6, reps: int = 3, seed: int = 7):
    """A timer that applies a seeded random circuit (the bench family) with the
    given knobs and returns the mean seconds per apply (CUDA events)."""
    import torch

    from . import workloads as W

    gates = W.random_layers(n_qubits, layers, seed=seed, mixed=True)
    stream = torch.cuda.Stream()
    sv = capi.Statevector(n_qubits, dtype, stream=stream.cuda_stream)

    def timer(knobs: dict) -> float:
        set_knobs(knobs)
        sv.set_basis(0)
        sv.apply(gates)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            sv.set_basis(0)
            sv.apply(gates)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps / 1e3

    timer.close = sv.close  # type: ignore[attr-defined]
    return timer


def load(n_qubits: int, dtype: int = capi.KT_C128, path: pathlib.Path | None = None,
         device: str | None = None) -> dict | None:
    """Set and return the cached knobs for this GPU, dtype and size (None if absent)."""
    p = path or cache_path()
    if not p.exists():
        return None
    data = json.loads(p.read_text())
    hit = data.get(_key(device or _device_name(), dtype, n_qubits))
    if hit:
        set_knobs(hit["knobs"])
        return hit["knobs"]
    return None


def save(n_qubits: int, dtype: int, knobs: dict, table: list, path: pathlib.Path | None = None,
         device: str | None = None) -> None:
    p = path or cache_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    data = json.loads(p.read_text()) if p.exists() else {}
    data[_key(device or _device_name(), dtype, n_qubits)] = {"knobs": knobs, "table": table, "when": time.time()}
    p.write_text(json.dumps(data, indent=1, sort_keys=True))


def autotune(n_qubits: int, dtype: int = capi.KT_C128, tune_qubits: int | None = None, grid: dict | None = None,
             use_cache: bool = True, path: pathlib.Path | None = None, timer=None) -> dict:
    """Pick and set the fastest knobs for `n_qubits`.

    The timing runs at `tune_qubits` (default min(n_qubits, 26): one tile pass
    behaves the same at every size above the tile, and a 26-qubit state keeps
    the search to seconds).  With `use_cache`, a cached answer is reused and a
    new one stored."""
    if use_cache:
        hit = load(n_qubits, dtype, path)
        if hit is not None:
            return hit
    nq = tune_qubits or min(n_qubits, 26)
    own = timer is None
    if own:
        timer = gpu_timer(nq, dtype)
    saved = current()

    def timed(knobs: dict) -> float:
        set_knobs(knobs)
        return timer(knobs)

    try:
        best, table = search(timed, candidates(grid))
    finally:
        set_knobs(saved)
        if own:
            timer.close()
    set_knobs(best)
    if use_cache:
        save(n_qubits, dtype, best, table, path)
    return best


# ---------------------------------------------------------------------------
# Batches (kt_batch).  A batch reads its knobs when it is created: which HBM
# items run the compiled class kernels (`batch_jit_min_qubits`, 0 = none: the
# persistent kernel's interpreted blocks), how large an item may be to run
# whole in shared memory (`batch_small_max_qubits`), and the fusion depth of
# its blocks (`fused_max_ops`).  The tile is the 256-thread CTA's.  Every
# candidate computes the same energies and gradients up to FP64 rounding.

BATCH_KNOBS = ("batch_jit_min_qubits", "batch_small_max_qubits", "fused_max_ops")
BATCH_GRID = {
    "batch_jit_min_qubits": (13, 16, 0),
    "batch_small_max_qubits": (13, 12),
    "fused_max_ops": (128, 256),
}


def batch_candidates(grid: dict | None = None) -> list[dict]:
    """All batch knob combinations of `grid` (defaults to BATCH_GRID), in a fixed order."""
    g = dict(BATCH_GRID)
    if grid:
        g.update(grid)
    return [dict(zip(BATCH_KNOBS, combo)) for combo in itertools.product(*(g[k] for k in BATCH_KNOBS))]


def batch_gpu_timer(batch_args: tuple, params, dtype: int = capi.KT_C128, reps: int = 2):
    """A timer that creates the batch (`batch_args` as capi.batch_items returns
    them) with the given knobs, evaluates it once, and returns the mean seconds
    of `reps` more evaluations (CUDA events; creation and compilation are not
    timed)."""
    import torch

    items, gates, strings, coeffs, n_params = batch_args
    stream = torch.cuda.Stream()

    def timer(knobs: dict) -> float:
        set_knobs(knobs)
        b = capi.Batch(items, gates, strings, coeffs, n_params, dtype=dtype)
        try:
            b.set_stream(stream.cuda_stream)
            b.evaluate(params)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                b.evaluate(params)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps / 1e3
        finally:
            b.close()

    return timer


def autotune_batch(batch_args: tuple, params, dtype: int = capi.KT_C128, grid: dict | None = None,
                   use_cache: bool = True, path: pathlib.Path | None = None, timer=None) -> dict:
    """Pick and set the fastest batch knobs for this batch's shape.  The cache
    key is the GPU, the dtype and the item count with the largest item's qubits
    (`batch|<items>x<max qubits>` in place of a qubit count)."""
    items = batch_args[0]
    shape = f"batch|{len(items)}x{int(max(items['n_qubits']))}"
    if use_cache:
        hit = load(shape, dtype, path)  # type: ignore[arg-type]
        if hit is not None:
            return hit
    own = timer is None
    if own:
        timer = batch_gpu_timer(batch_args, params, dtype)
    saved = {k: capi.tuning_get(k) for k in BATCH_KNOBS}

    def timed(knobs: dict) -> float:
        set_knobs(knobs)
        return timer(knobs)

    try:
        best, table = search(timed, batch_candidates(grid))
    finally:
        set_knobs(saved)
    set_knobs(best)
    if use_cache:
        save(shape, dtype, best, table, path)  # type: ignore[arg-type]
    return best
