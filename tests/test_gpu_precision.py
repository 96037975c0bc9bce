"""complex64 storage with FP64 reductions: every fused block rescales to the
norm the state had when the apply began, so the norm does not drift with the
FP32 rounding of thousands of gates, unnormalised inputs keep their norm, and
the state stays within FP32 rounding of the complex128 oracle."""
import numpy as np
import pytest

from conftest import basis, random_state
from kettle_b200 import capi
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _c64_state(n, gates, renorm, upload=None):
    old = capi.tuning_get("c64_renormalize")
    capi.tuning_set("c64_renormalize", 1 if renorm else 0)
    try:
        sv = capi.Statevector(n, capi.KT_C64)
        if upload is not None:
            sv.upload(upload)
        sv.apply(gates)
        out = sv.download(), sv.norm_sq()
        sv.close()
    finally:
        capi.tuning_set("c64_renormalize", old)
    return out


def test_renormalised_c64_keeps_the_norm(engine, port):
    n = 16
    gates = W.random_layers(n, 150, seed=5, mixed=True)
    want = port.apply(n, basis(n), gates)
    a1, n1 = _c64_state(n, gates, renorm=True)
    a0, n0 = _c64_state(n, gates, renorm=False)
    assert abs(n1 - 1.0) < 1e-6
    assert abs(n1 - 1.0) <= abs(n0 - 1.0)
    assert np.abs(a1 - want).max() < 1e-4
    assert np.abs(a0 - want).max() < 1e-4


def test_renormalised_c64_keeps_an_unnormalised_input(engine, port):
    n = 14
    gates = W.random_layers(n, 60, seed=6, mixed=True)
    psi0 = 0.5 * random_state(n, 6)
    want = port.apply(n, psi0, gates)
    a, nrm = _c64_state(n, gates, renorm=True, upload=psi0)
    assert abs(nrm - 0.25) < 0.25 * 1e-6
    assert np.abs(a - want).max() < 1e-4


def test_c64_density_matrix(engine, port):
    n = 6
    g = W.random_layers(n, 20, seed=8, mixed=True)
    dm = capi.DensityMatrix(n, capi.KT_C64)
    dm.apply(g)
    rho = dm.download()
    rho0 = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    rho0[0, 0] = 1
    want = port.simulate_dm(n, rho0, g)
    assert np.abs(rho - want).max() < 1e-4
    assert abs(dm.trace() - 1.0) < 1e-5
