"""The bench's CPU baselines, run on the host without a GPU: the batch
baseline's processes (spawned, each timing the same bounded sample through the
reference library) and the scaling of their figures to a whole batch."""
import numpy as np
import pytest

from kettle_b200 import workloads as W


def test_batch_cpu_reference_scales_the_sample(ref):
    import bench

    circuits, _ = W.hea_batch(24, seed=5, qubits=(10, 12), layers=(2, 3))
    out = bench.batch_cpu_reference(circuits, processes=2)
    assert out["processes"] == 2 and out["kind"] == "reference" and out["unit"] == "instances/s"
    qs = sorted({c[0] for c in circuits})
    assert sorted(out["seconds_per_layer_process0"]) == qs
    assert all(v > 0 for v in out["seconds_per_layer_process0"].values())
    assert all(v > 0 for v in out["seconds_per_term_process0"].values())
    # the gradient costs 1 + 2 P evaluations of the energy per instance
    P_min = min(c[2] for c in circuits)
    assert out["instances_per_s"] < out["energy_only_instances_per_s"] / (1 + 2 * P_min) * 1.0001
    # two processes: the host rate is the sum of two single-process rates,
    # each of them the batch size over that process's scaled time
    layer = out["seconds_per_layer_process0"]
    term = out["seconds_per_term_process0"]
    t_e = sum(round(int((g["op"] == W.gate("CZ", 1)["op"][0]).sum()) / n) * layer[n] + s.size * term[n]
              for n, g, p, s, c in circuits)
    one = len(circuits) / t_e
    assert 0.2 * 2 * one < out["energy_only_instances_per_s"] < 5 * 2 * one


def test_batch_ref_strings_bounds():
    import bench

    assert bench._batch_ref_strings(10) == 50
    assert bench._batch_ref_strings(22) == 2
    counts = [bench._batch_ref_strings(n) for n in range(10, 23)]
    assert counts == sorted(counts, reverse=True)
    assert np.all(np.array(counts) >= 2)


@pytest.mark.parametrize("n", [10, 16])
def test_batch_sample_layer_is_one_ansatz_layer(n):
    """The timed layer is the ansatz's first layer: RY and RZ on every qubit,
    then the n CZ gates of the ring."""
    from kettle_b200.capi import OP

    gates, _ = W.hea(n, 3, seed=1)
    ops = gates["op"].astype(int)
    cz = np.flatnonzero(ops == OP["CZ"])
    end = int(cz[n - 1]) + 1
    assert end == 3 * n
    assert (ops[:n] == OP["RY"]).all() and (ops[n:2 * n] == OP["RZ"]).all() and (ops[2 * n:end] == OP["CZ"]).all()
