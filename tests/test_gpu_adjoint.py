"""Adjoint gradients on the GPU, through the C-ABI.

Checked against central finite differences (step 1e-5) of the oracle's own
forward + expectation value, and against the parameter-shift rule evaluated
with the engine's forward passes (RX/RY/RZ: [E(t + pi/2) - E(t - pi/2)] / 2).
Tolerance: max |d grad| <= 1e-8 against finite differences, 1e-10 against
parameter shift (both complex128)."""
import math

import numpy as np
import pytest

from conftest import basis
from kettle_b200 import capi
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu


def energy_oracle(port, n, gates, params, strings, coeffs):
    psi = port.apply(n, basis(n), gates, params)
    _, total = port.expect(n, psi, strings, coeffs)
    return total.real


def engine_energy(n, gates, params, strings, coeffs, dtype=capi.KT_C128):
    sv = capi.Statevector(n, dtype)
    sv.apply(gates, params)
    _, total = sv.expect(strings, coeffs)
    sv.close()
    return total.real


def adjoint(n, gates, params, strings, coeffs, checkpoint=0, dtype=capi.KT_C128):
    sv = capi.Statevector(n, dtype)
    adj = capi.Adjoint(sv, checkpoint)
    e = adj.forward(gates, params, strings, coeffs)
    g = adj.backward()
    back = sv.download()
    adj.close()
    sv.close()
    return e, g, back


@pytest.mark.parametrize("n,layers", [(6, 2), (9, 3)])
def test_adjoint_vs_finite_differences(engine, port, n, layers):
    gates, params = W.hea(n, layers, seed=n)
    strings, coeffs = W.xxz_chain(n, seed=n)
    e, g, back = adjoint(n, gates, params, strings, coeffs)
    assert abs(e - energy_oracle(port, n, gates, params, strings, coeffs)) < 1e-12
    h = 1e-5
    fd = np.zeros_like(params)
    for k in range(params.size):
        pp, pm = params.copy(), params.copy()
        pp[k] += h
        pm[k] -= h
        fd[k] = (energy_oracle(port, n, gates, pp, strings, coeffs) -
                 energy_oracle(port, n, gates, pm, strings, coeffs)) / (2 * h)
    assert np.abs(g - fd).max() < 1e-8
    # the backward sweep un-applies the circuit: psi is back at |0...0>
    assert abs(back[0] - 1) < 1e-12 and np.abs(back[1:]).max() < 1e-12


def test_adjoint_vs_parameter_shift(engine):
    n = 10
    gates, params = W.hea(n, 3, seed=3)
    strings, coeffs = W.random_paulis(n, 30, seed=3)
    coeffs = coeffs.real.astype(np.complex128)
    _, g, _ = adjoint(n, gates, params, strings, coeffs)
    ps = np.zeros_like(params)
    for k in range(params.size):
        pp, pm = params.copy(), params.copy()
        pp[k] += math.pi / 2
        pm[k] -= math.pi / 2
        ps[k] = 0.5 * (engine_energy(n, gates, pp, strings, coeffs) - engine_energy(n, gates, pm, strings, coeffs))
    assert np.abs(g - ps).max() < 1e-10


def test_adjoint_shared_and_controlled_parameters(engine, port):
    n = 7
    rng = np.random.default_rng(5)
    recs = []
    for q in range(n):
        recs.append(W.gate("RX", q, param=q % 3))      # three shared parameters
    for q in range(n - 1):
        recs.append(W.gate("CRY", q + 1, control=q, param=3))
        recs.append(W.gate("CP", q, control=q + 1, param=4))
        recs.append(W.gate("CRZ", (q + 2) % n, control=q, param=5))
        recs.append(W.gate("H", q))
        recs.append(W.gate("CRX", q, control=(q + 3) % n, param=6))
        recs.append(W.gate("P", q, param=7))
        recs.append(W.gate("U", q, u=W.haar_unitary2(rng)))
    gates = np.concatenate(recs)
    params = rng.uniform(-math.pi, math.pi, 8)
    strings, coeffs = W.random_paulis(n, 20, seed=6)
    coeffs = coeffs.real.astype(np.complex128)
    _, g, _ = adjoint(n, gates, params, strings, coeffs)
    h = 1e-5
    fd = np.array([(energy_oracle(port, n, gates, params + h * np.eye(8)[k], strings, coeffs) -
                    energy_oracle(port, n, gates, params - h * np.eye(8)[k], strings, coeffs)) / (2 * h)
                   for k in range(8)])
    assert np.abs(g - fd).max() < 1e-8


def test_adjoint_checkpoints_match(engine):
    n = 12
    gates, params = W.hea(n, 4, seed=8)
    strings, coeffs = W.xxz_chain(n, seed=8)
    e0, g0, _ = adjoint(n, gates, params, strings, coeffs, checkpoint=0)
    e1, g1, _ = adjoint(n, gates, params, strings, coeffs, checkpoint=16)
    # each checkpoint segment is planned on its own, so gates on disjoint
    # qubits may run in another (equally valid) order: equal to rounding
    assert abs(e0 - e1) < 1e-13
    assert np.abs(g0 - g1).max() < 1e-12


def test_adjoint_complex64(engine):
    n = 12
    gates, params = W.hea(n, 3, seed=9)
    strings, coeffs = W.xxz_chain(n, seed=9)
    e0, g0, _ = adjoint(n, gates, params, strings, coeffs)
    e1, g1, _ = adjoint(n, gates, params, strings, coeffs, dtype=capi.KT_C64)
    assert abs(e0 - e1) < 1e-4
    assert np.abs(g0 - g1).max() < 1e-3
