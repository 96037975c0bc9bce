"""Every autotuner candidate computes the same state (the knobs only regroup
gates into blocks), and autotune() leaves the fastest candidate set."""
import numpy as np
import pytest

from conftest import basis
from kettle_b200 import autotune as AT
from kettle_b200 import capi
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,tol", [(capi.KT_C128, 1e-12), (capi.KT_C64, 1e-4)])
def test_candidates_agree(engine, port, dtype, tol):
    n = 16
    gates = W.random_layers(n, 6, seed=3, mixed=True)
    want = port.apply(n, basis(n), gates)
    before = AT.current()
    try:
        for knobs in AT.candidates():
            AT.set_knobs(knobs)
            sv = capi.Statevector(n, dtype)
            sv.apply(gates)
            assert np.abs(sv.download() - want).max() < tol, knobs
            sv.close()
    finally:
        AT.set_knobs(before)


def test_autotune_on_device(engine, tmp_path):
    before = AT.current()
    try:
        grid = {"fused_tile_bits": (11, 12), "fused_max_ops": (128, 256), "fused_ctas_per_sm": (2,)}
        best = AT.autotune(20, grid=grid, path=tmp_path / "t.json")
        assert AT.current() == best
        assert AT.load(20, path=tmp_path / "t.json") == best
    finally:
        AT.set_knobs(before)


def test_batch_autotune_on_device(engine, tmp_path):
    """autotune_batch over compiled classes on / off and two fusion depths on a
    small mixed batch: every candidate gives the same energies and gradients
    (1e-11), the fastest is left set and cached."""
    circuits, params = W.hea_batch(24, seed=9, qubits=(11, 16), layers=(2, 4), n_strings=8)
    args = capi.batch_items(circuits)
    before = {k: capi.tuning_get(k) for k in AT.BATCH_KNOBS}
    grid = {"batch_jit_min_qubits": (13, 0), "batch_small_max_qubits": (12,), "fused_max_ops": (128, 256)}
    results = []
    try:
        for knobs in AT.batch_candidates(grid):
            AT.set_knobs(knobs)
            b = capi.Batch(*args)
            results.append(b.evaluate(params))
            b.close()
        for e, g in results[1:]:
            assert np.abs(e - results[0][0]).max() < 1e-11 and np.abs(g - results[0][1]).max() < 1e-11
        best = AT.autotune_batch(args, params, grid=grid, path=tmp_path / "b.json")
        assert {k: capi.tuning_get(k) for k in AT.BATCH_KNOBS} == best
        assert AT.load(f"batch|24x{int(max(args[0]['n_qubits']))}", capi.KT_C128, path=tmp_path / "b.json") == best
    finally:
        AT.set_knobs(before)
