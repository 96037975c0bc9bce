"""Sharded Pauli strings and parameter shifts on the engine (one GPU): the
ranks' shares of a 20-qubit state's 120 strings, evaluated with kt_sv_expect
and assembled, equal the unsharded terms and total; the sharded
parameter-shift gradient of an 8-qubit ansatz equals the adjoint gradient.
The collective itself is covered by the gloo tests (tests/test_distributed.py)."""
import numpy as np
import pytest

from kettle_b200 import capi
from kettle_b200 import distributed as D
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_sharded_strings_on_the_engine(engine):
    n = 20
    sv = capi.Statevector(n)
    sv.apply(W.random_layers(n, 3, seed=21, mixed=True))
    strings, coeffs = W.random_paulis(n, 120, seed=22)
    strings[60:90]["x"] = strings[0]["x"]  # a large X-mask group
    want_terms, want_total = sv.expect(strings, coeffs)
    world = 3
    terms = np.zeros(strings.size, dtype=np.complex128)
    for rank in range(world):
        t, _ = D.sharded_expectation(lambda s, c: sv.expect(s, c)[0], strings, coeffs, rank, world)
        terms += t  # without a process group each rank's vector holds only its own strings
    assert np.abs(terms - want_terms).max() < 1e-12
    assert abs(np.sum(coeffs * terms) - want_total) < 1e-11
    sv.close()


def test_sharded_parameter_shift_equals_adjoint(engine):
    n = 8
    gates, params = W.hea(n, 2, seed=23)
    strings, coeffs = W.xxz_chain(n, seed=23)
    sv = capi.Statevector(n)
    adj = capi.Adjoint(sv)
    adj.forward(gates, params, strings, coeffs)
    g_adj = adj.backward()
    adj.close()

    def energy(p):
        sv.set_basis(0)
        sv.apply(gates, p)
        return sv.expect(strings, coeffs)[1].real

    world = 2
    g = sum(D.sharded_parameter_shift(energy, params, rank, world) for rank in range(world))
    assert np.abs(g - g_adj).max() < 1e-10
    sv.close()
