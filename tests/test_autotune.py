"""Autotuner host logic (CPU): candidate grid, search, cache round trip, and
that the knobs it sets reach the library."""
import json

import pytest

from kettle_b200 import autotune as AT
from kettle_b200 import capi


def test_candidates_cover_the_grid_in_order():
    c = AT.candidates({"fused_tile_bits": (11, 12), "fused_max_ops": (128,), "fused_ctas_per_sm": (1, 2)})
    assert c == [
        {"fused_tile_bits": 11, "fused_max_ops": 128, "fused_ctas_per_sm": 1},
        {"fused_tile_bits": 11, "fused_max_ops": 128, "fused_ctas_per_sm": 2},
        {"fused_tile_bits": 12, "fused_max_ops": 128, "fused_ctas_per_sm": 1},
        {"fused_tile_bits": 12, "fused_max_ops": 128, "fused_ctas_per_sm": 2},
    ]
    assert len(AT.candidates()) == 24


def test_search_picks_fastest_and_keeps_first_on_ties():
    cands = AT.candidates({"fused_tile_bits": (10, 11, 12), "fused_max_ops": (64,), "fused_ctas_per_sm": (2,)})
    cost = {10: 3.0, 11: 1.0, 12: 1.0}
    best, table = AT.search(lambda k: cost[k["fused_tile_bits"]], cands)
    assert best["fused_tile_bits"] == 11
    assert [r["seconds"] for r in table] == [3.0, 1.0, 1.0]


def test_autotune_sets_caches_and_restores(tmp_path):
    path = tmp_path / "t.json"
    before = AT.current()
    seen = []

    def fake(knobs):
        seen.append(dict(knobs))
        assert AT.current() == knobs  # the knobs are live while timed
        return 1.0 / knobs["fused_max_ops"] + (0.0 if knobs["fused_ctas_per_sm"] == 2 else 1.0)

    grid = {"fused_tile_bits": (12,), "fused_max_ops": (64, 256), "fused_ctas_per_sm": (1, 2)}
    best = AT.autotune(24, capi.KT_C128, grid=grid, path=path, timer=fake, use_cache=False)
    assert best == {"fused_tile_bits": 12, "fused_max_ops": 256, "fused_ctas_per_sm": 2}
    assert AT.current() == best
    assert len(seen) == 4
    AT.save(24, capi.KT_C128, best, [], path=path, device="fake-gpu")
    AT.set_knobs(before)
    assert AT.load(24, capi.KT_C128, path=path, device="fake-gpu") == best
    assert AT.current() == best
    assert AT.load(25, capi.KT_C128, path=path, device="fake-gpu") is None
    data = json.loads(path.read_text())
    assert "fake-gpu|c128|24" in data
    AT.set_knobs(before)


def test_unknown_knob_is_rejected():
    with pytest.raises(capi.KettleError):
        capi.tuning_set("no_such_knob", 1)


def test_batch_autotune_picks_sets_and_caches(tmp_path):
    """The batch grid (compiled-class threshold, shared-memory limit, fusion
    depth): every candidate is live while timed, the fastest is left set, the
    table is cached under the batch's shape key, and the previous knobs can be
    restored."""
    import numpy as np
    before = {k: capi.tuning_get(k) for k in AT.BATCH_KNOBS}
    items = np.zeros(3, dtype=capi.BATCH_ITEM_DTYPE)
    items["n_qubits"] = [12, 18, 20]
    seen = []

    def fake(knobs):
        seen.append(dict(knobs))
        assert {k: capi.tuning_get(k) for k in AT.BATCH_KNOBS} == knobs
        return (2.0 if knobs["batch_jit_min_qubits"] == 0 else 1.0) + (0.5 if knobs["fused_max_ops"] == 128 else 0.0)

    grid = {"batch_jit_min_qubits": (0, 16), "batch_small_max_qubits": (13,), "fused_max_ops": (128, 256)}
    path = tmp_path / "b.json"
    best = AT.autotune_batch((items, None, None, None, 0), None, capi.KT_C128, grid=grid, timer=fake, use_cache=False)
    assert best == {"batch_jit_min_qubits": 16, "batch_small_max_qubits": 13, "fused_max_ops": 256}
    assert len(seen) == 4 and len(AT.batch_candidates()) == 12
    assert {k: capi.tuning_get(k) for k in AT.BATCH_KNOBS} == best
    AT.save("batch|3x20", capi.KT_C128, best, [], path=path, device="fake-gpu")
    assert "fake-gpu|c128|batch|3x20" in json.loads(path.read_text())
    AT.set_knobs(before)
