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
