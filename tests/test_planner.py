"""The fused-block planner is host logic: it runs here without a GPU
(kt_plan_stats).  Every gate must land in exactly one block, the block count
must drop well below the gate count on the benchmark circuits, the plan
must react to the tuning knobs, and the order in which it runs the gates
(kt_plan_order) must keep every pair of gates sharing a qubit in order."""
import time

import numpy as np
import pytest

from kettle_b200 import capi
from kettle_b200 import workloads as W


def test_every_gate_is_planned_once():
    for n, layers, mixed in ((10, 6, True), (16, 4, True), (22, 3, False), (30, 2, True)):
        g = W.random_layers(n, layers, seed=n, mixed=mixed)
        st = capi.plan_stats(n, g)
        assert st["ops"] == len(g)
        assert 1 <= st["blocks"] <= len(g)
        assert st["phases"] >= st["blocks"]


def test_small_states_use_per_gate_sweeps():
    g = W.random_layers(8, 3, seed=1)
    assert capi.plan_stats(8, g) == {"blocks": 0, "phases": 0, "ops": 0, "transposes": 0}


def test_fusion_depth_on_benchmark_circuit():
    g = W.random_layers(30, 40, seed=2024, mixed=True)
    t0 = time.perf_counter()
    st = capi.plan_stats(30, g)
    dt = time.perf_counter() - t0
    assert st["blocks"] < len(g) / 15          # at least ~15 gates per HBM pass
    assert dt < 2.0                            # planning is cheap next to a 30-qubit step
    c64 = capi.plan_stats(30, g, dtype=capi.KT_C64)
    assert c64["blocks"] <= st["blocks"]       # one more tile qubit for complex64


def test_tuning_knobs_change_the_plan():
    g = W.random_layers(26, 6, seed=3, mixed=True)
    base = capi.plan_stats(26, g)
    old = capi.tuning_get("fused_max_ops")
    try:
        capi.tuning_set("fused_max_ops", 8)
        small = capi.plan_stats(26, g)
    finally:
        capi.tuning_set("fused_max_ops", old)
    assert small["blocks"] >= len(g) // 8
    assert small["blocks"] > base["blocks"]
    assert capi.plan_stats(26, g) == base


def test_diagonal_gates_cost_no_tile_qubit():
    # a long run of diagonal gates on every qubit fits in a single block
    n = 24
    recs = [W.gate("RZ", q, angle=0.1 * q) for q in range(n)] + [W.gate("CZ", (q + 1) % n, control=q) for q in range(n)]
    st = capi.plan_stats(n, np.concatenate(recs))
    assert st["blocks"] == 1


def test_lookahead_takes_fewer_passes():
    # pinning a block's tile to the qubits the next gates need most (with a
    # two-block lookahead) never costs passes on these circuits and saves some
    cases = [(30, W.random_layers(30, 40, seed=2024, mixed=True)), (26, W.random_layers(26, 20, seed=5, mixed=False)),
             (28, W.random_layers(28, 30, seed=7, mixed=True))]
    old = capi.tuning_get("plan_lookahead")
    try:
        saved = 0
        for n, g in cases:
            capi.tuning_set("plan_lookahead", 0)
            greedy = capi.plan_stats(n, g)
            capi.tuning_set("plan_lookahead", 1)
            look = capi.plan_stats(n, g)
            assert look["ops"] == greedy["ops"] == len(g)
            assert look["blocks"] <= greedy["blocks"]
            saved += greedy["blocks"] - look["blocks"]
        assert saved > 0
    finally:
        capi.tuning_set("plan_lookahead", old)


def _keeps_dependencies(gates, order):
    # every pair of gates sharing a qubit takes effect in the given order
    controlled = {capi.OP[x] for x in capi.CONTROLLED}
    last = {}
    for i in order:
        g = gates[int(i)]
        qs = (int(g["target"]), int(g["control"])) if int(g["op"]) in controlled else (int(g["target"]),)
        for q in qs:
            if last.get(q, -1) > i:
                return False
            last[q] = max(last.get(q, -1), int(i))
    return True


PLAN_CASES = [(30, W.random_layers(30, 40, seed=2024, mixed=True), None),
              (26, W.random_layers(26, 20, seed=5, mixed=False), None),
              (28, W.random_layers(28, 30, seed=7, mixed=True), None),
              (30, *W.hea(30, 8, seed=1)), (24, *W.hea(24, 6, seed=3))]


@pytest.mark.parametrize("schedule", [0, 1, 2, 3])
def test_plan_order_is_a_dependency_order(schedule):
    # blocks take gates ahead of earlier gates on disjoint qubits, and with
    # plan_schedule = 1 a block's gates run in any order that saves
    # transposes: every gate exactly once, gates sharing a qubit in order
    old = capi.tuning_get("plan_schedule")
    try:
        capi.tuning_set("plan_schedule", schedule)
        for n, g, p in PLAN_CASES + [(18, W.random_layers(18, 12, seed=77, mixed=True), None)]:
            order = capi.plan_order(n, g, p)
            assert sorted(order.tolist()) == list(range(len(g)))
            assert _keeps_dependencies(g, order)
        assert capi.plan_order(8, W.random_layers(8, 2, seed=1)).size == 0
    finally:
        capi.tuning_set("plan_schedule", old)


def test_plan_order_catches_a_swapped_pair():
    # the dependency check itself: two gates on one qubit swapped is caught
    g = np.concatenate([W.gate("H", 3), W.gate("RX", 5, angle=0.2), W.gate("CX", 5, control=3)])
    assert _keeps_dependencies(g, [0, 1, 2]) and _keeps_dependencies(g, [1, 0, 2])
    assert not _keeps_dependencies(g, [2, 0, 1]) and not _keeps_dependencies(g, [0, 2, 1])


def test_list_scheduling_takes_fewer_transposes():
    # running ready gates that fit the current register set before a
    # transpose saves transposes on every case and changes no block; choosing
    # each new register set by the gates it takes saves a few more
    old = capi.tuning_get("plan_schedule")
    try:
        for n, g, p in PLAN_CASES:
            capi.tuning_set("plan_schedule", 0)
            given = capi.plan_stats(n, g, p)
            capi.tuning_set("plan_schedule", 1)
            sched = capi.plan_stats(n, g, p)
            assert sched["blocks"] == given["blocks"] and sched["ops"] == given["ops"] == len(g)
            assert sched["transposes"] < given["transposes"]
            # register sets chosen by the gates they take: never more transposes here
            capi.tuning_set("plan_schedule", 2)
            gain = capi.plan_stats(n, g, p)
            assert gain["blocks"] == given["blocks"] and gain["ops"] == len(g)
            assert gain["transposes"] <= sched["transposes"]
            # a first register set above the 128-byte run bits: no more here either
            capi.tuning_set("plan_schedule", 3)
            high = capi.plan_stats(n, g, p)
            assert high["blocks"] == given["blocks"] and high["ops"] == len(g)
            assert high["transposes"] <= gain["transposes"]
        # the 30-qubit bench circuit: 379 -> 251 -> 243 -> 239
        assert capi.plan_stats(*PLAN_CASES[0][:2])["transposes"] <= 0.65 * 379
    finally:
        capi.tuning_set("plan_schedule", old)
