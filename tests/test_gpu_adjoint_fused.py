"""The fused adjoint sweep against the one-kernel-per-gate sweep and finite
differences: same gradients (1e-11), with and without forward checkpoints,
on circuits whose gates the planner reorders across blocks."""
import numpy as np
import pytest

from conftest import basis
from kettle_b200 import capi
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _grad(n, gates, params, strings, coeffs, fused, checkpoint=0, dtype=capi.KT_C128):
    old = capi.tuning_get("adjoint_fused")
    capi.tuning_set("adjoint_fused", 1 if fused else 0)
    try:
        sv = capi.Statevector(n, dtype)
        adj = capi.Adjoint(sv, checkpoint)
        e = adj.forward(gates, params, strings, coeffs)
        g = adj.backward()
        back = sv.download()
        adj.close()
        sv.close()
    finally:
        capi.tuning_set("adjoint_fused", old)
    return e, g, back


def _mixed_param_circuit(n, seed):
    rng = np.random.default_rng(seed)
    recs, slot = [], 0
    names = ["RX", "RY", "RZ", "P", "CRX", "CRY", "CRZ", "CP"]
    for layer in range(4):
        for q in range(n):
            name = names[int(rng.integers(4))]
            recs.append(W.gate(name, q, param=slot))
            slot += 1
        for _ in range(n // 2):
            c, t = rng.choice(n, 2, replace=False)
            name = names[4 + int(rng.integers(4))]
            recs.append(W.gate(name, int(t), control=int(c), param=slot))
            slot += 1
        for q in range(layer % 2, n - 1, 2):
            recs.append(W.gate("CX", q + 1, control=q))
        recs.append(W.gate("U", int(rng.integers(n)), u=W.haar_unitary2(rng)))
        recs.append(W.gate("H", int(rng.integers(n))))
    params = rng.uniform(-np.pi, np.pi, slot)
    params[::7] = params[3]  # a few shared values (separate slots)
    return np.concatenate(recs), params


@pytest.mark.parametrize("n", [9, 13, 17])
def test_fused_equals_per_gate(engine, n):
    gates, params = _mixed_param_circuit(n, n)
    strings, coeffs = W.random_paulis(n, 40, seed=n)
    coeffs = coeffs.real.astype(np.complex128)
    e0, g0, b0 = _grad(n, gates, params, strings, coeffs, fused=False)
    e1, g1, b1 = _grad(n, gates, params, strings, coeffs, fused=True)
    assert e0 == e1
    assert np.abs(g0 - g1).max() < 1e-11
    assert abs(b1[0] - 1) < 1e-11 and np.abs(b1[1:]).max() < 1e-11


def test_fused_vs_finite_differences(engine, port):
    n = 10
    gates, params = W.hea(n, 3, seed=7)
    gates = np.concatenate([gates, W.gate("CRY", 3, control=8, param=5), W.gate("CP", 0, control=9, param=11)])
    strings, coeffs = W.xxz_chain(n, seed=7)
    _, g, _ = _grad(n, gates, params, strings, coeffs, fused=True)
    h = 1e-5

    def energy(p):
        psi = port.apply(n, basis(n), gates, p)
        return port.expect(n, psi, strings, coeffs)[1].real

    fd = np.array([(energy(params + h * np.eye(params.size)[k]) - energy(params - h * np.eye(params.size)[k])) / (2 * h)
                   for k in range(params.size)])
    assert np.abs(g - fd).max() < 1e-8


@pytest.mark.parametrize("checkpoint", [7, 40])
def test_fused_with_checkpoints(engine, checkpoint):
    n = 14
    gates, params = W.hea(n, 5, seed=2)
    strings, coeffs = W.xxz_chain(n, seed=2)
    _, g0, _ = _grad(n, gates, params, strings, coeffs, fused=False)
    _, g1, _ = _grad(n, gates, params, strings, coeffs, fused=True, checkpoint=checkpoint)
    assert np.abs(g0 - g1).max() < 1e-11


def test_fused_complex64(engine):
    n = 13
    gates, params = W.hea(n, 3, seed=3)
    strings, coeffs = W.xxz_chain(n, seed=3)
    _, g0, _ = _grad(n, gates, params, strings, coeffs, fused=True)
    _, g1, _ = _grad(n, gates, params, strings, coeffs, fused=True, dtype=capi.KT_C64)
    assert np.abs(g0 - g1).max() < 1e-3


def test_fused_deep_blocks(engine):
    """A deep ansatz whose adjoint blocks hit the per-block op cap (shared-memory budget)."""
    n = 16
    gates, params = W.hea(n, 10, seed=4)
    strings, coeffs = W.xxz_chain(n, seed=4)
    e0, g0, _ = _grad(n, gates, params, strings, coeffs, fused=False)
    e1, g1, _ = _grad(n, gates, params, strings, coeffs, fused=True)
    assert e0 == e1
    assert np.abs(g0 - g1).max() < 1e-11


def _with_adjoint_jit(mode, fn):
    old = capi.tuning_get("adjoint_jit")
    capi.tuning_set("adjoint_jit", mode)
    try:
        return fn()
    finally:
        capi.tuning_set("adjoint_jit", old)


@pytest.mark.parametrize("n,dtype,checkpoint", [(9, capi.KT_C128, 0), (13, capi.KT_C128, 0), (17, capi.KT_C128, 0),
                                                (14, capi.KT_C128, 25), (13, capi.KT_C64, 0)])
def test_compiled_adjoint_blocks_equal_interpreted(engine, n, dtype, checkpoint):
    """Run-time compiled adjoint blocks (adjoint_jit = 1: gradient terms and
    U^dagger bodies as straight-line code) against the interpreted fused
    blocks (adjoint_jit = 0): the same energy and gradient (1e-12; complex64
    1e-5), the state un-applied back to |0...0>; repeated with new parameters
    (plan cache, kernels reused)."""
    gates, params = _mixed_param_circuit(n, 100 + n)
    strings, coeffs = W.random_paulis(n, 30, seed=n)
    coeffs = coeffs.real.astype(np.complex128)
    tol = 1e-12 if dtype == capi.KT_C128 else 1e-5
    for shift in (0.0, 0.37):
        p = params + shift
        e0, g0, _ = _with_adjoint_jit(0, lambda: _grad(n, gates, p, strings, coeffs, True, checkpoint, dtype))
        s0 = capi.jit_stats()
        e1, g1, b1 = _with_adjoint_jit(1, lambda: _grad(n, gates, p, strings, coeffs, True, checkpoint, dtype))
        s1 = capi.jit_stats()
        assert not s1["failed"] and s1["launches"] > s0["launches"]
        assert abs(e0 - e1) < tol
        assert np.abs(g0 - g1).max() < tol
        assert abs(b1[0] - 1) < 10 * tol and np.abs(b1[1:]).max() < 10 * tol
