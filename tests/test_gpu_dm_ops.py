"""Density-matrix operations on the GPU (kt_dm_partial_trace, kt_dm_tensor_product,
kt_dm_trace_of_square) against the reference's outputs (tests/golden/golden_dm_ops.npz)
and the oracle on seeded inputs up to 12 qubits; and a density matrix whose
circuit was compiled ahead (kt_dm_prepare).

Partial traces add the same values in the same grouping as the reference's
one-qubit-at-a-time sequence (state/density_matrix.cpp:231-278), so complex128
results are bit-identical; products (tensor product, Tr(rho^2)) may contract
to FMA on the device and are held to 1e-15 / 1e-13; complex64 storage to 1e-6."""
import numpy as np
import pytest

from conftest import GOLDEN
from kettle_b200 import capi

pytestmark = pytest.mark.gpu


def _rho(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((1 << n, 1 << n)) + 1j * rng.standard_normal((1 << n, 1 << n))
    rho = a @ a.conj().T
    return rho / np.trace(rho)


def _dm(capi, rho, dtype=None):
    n = int(np.log2(rho.shape[0]))
    d = capi.DensityMatrix(n, capi.KT_C128 if dtype is None else dtype)
    d.upload(rho)
    return d


def _sequential_to_distinct(n, qubits):
    """The reference's reading of a traced-qubit list (sorted high to low, each
    an index into the matrix left so far) as distinct original qubits, in trace order."""
    remaining = list(range(n))
    out = []
    for p in sorted(qubits, reverse=True):
        out.append(remaining.pop(p))
    return out


def test_partial_trace_matches_reference_golden_bit_for_bit(engine):
    g = dict(np.load(GOLDEN / "golden_dm_ops.npz"))
    for n in (3, 4, 5):
        d = _dm(engine, g[f"dmop_{n}_rho"])
        j = 0
        while f"dmop_{n}_pt_{j}_q" in g:
            qs = _sequential_to_distinct(n, g[f"dmop_{n}_pt_{j}_q"].tolist())
            out = d.partial_trace(qs)
            assert out.n_qubits == n - len(qs)
            assert np.array_equal(out.download(), g[f"dmop_{n}_pt_{j}_out"]), (n, j)
            out.close()
            j += 1
        assert abs(d.trace_of_square() - g[f"dmop_{n}_tsq"][0]) < 1e-13
        d.close()
    left, right = _dm(engine, g["dmop_tp_left"]), _dm(engine, g["dmop_tp_right"])
    t = left.tensor_product(right)
    assert t.n_qubits == 5
    np.testing.assert_allclose(t.download(), g["dmop_tp_out"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("n,cases", [
    (8, [[0], [7], [3, 5], [7, 6, 5, 4], [0, 2, 4, 6]]),
    (10, [[9], [0], [1, 8, 4], list(range(10))]),
    (12, [[11], [0, 6], [2, 3, 4, 5, 6, 7, 8, 9, 10, 11]]),
])
def test_partial_trace_vs_oracle(engine, port, n, cases):
    rho = _rho(n, 50 + n)
    d = _dm(engine, rho)
    for qs in cases:
        want = port.dm_partial_trace(n, rho, qs)
        got = d.partial_trace(_sequential_to_distinct(n, qs))
        assert np.array_equal(got.download(), want), (n, qs)
        got.close()


def test_partial_trace_edge_cases(engine):
    rho = _rho(4, 9)
    d = _dm(engine, rho)
    # nothing traced: a copy
    same = d.partial_trace([])
    assert np.array_equal(same.download(), rho)
    # everything traced: a 1 x 1 matrix holding the trace
    one = d.partial_trace([3, 2, 1, 0])
    assert one.n_qubits == 0
    got = one.download()
    assert got.shape == (1, 1) and abs(got[0, 0] - np.trace(rho)) < 1e-14
    # a traced qubit out of range, a repeated one, or a wrong output size: errors, no launch
    for bad in ([4], [-1], [1, 1]):
        with pytest.raises(engine.KettleError):
            d.partial_trace(bad)
    out = engine.DensityMatrix(2)
    q = np.array([0], dtype=np.int32)
    with pytest.raises(engine.KettleError):
        engine.check(engine.lib().kt_dm_partial_trace(d._h, engine.ptr(q), 1, out._h))
    assert np.array_equal(d.download(), rho)


def test_tensor_product_and_purity_vs_oracle(engine, port):
    a, b = _rho(3, 1), _rho(5, 2)
    da, db = _dm(engine, a), _dm(engine, b)
    t = da.tensor_product(db)
    want = port.dm_tensor_product(3, a, 5, b)
    np.testing.assert_allclose(t.download(), want, rtol=0, atol=1e-15)
    # tracing the right factor's qubits leaves the left factor times Tr(b)
    back = t.partial_trace(list(range(7, 2, -1)))
    np.testing.assert_allclose(back.download(), a, rtol=0, atol=1e-14)
    for n, r in ((3, a), (5, b), (8, want)):
        d = _dm(engine, r)
        assert abs(d.trace_of_square() - port.dm_trace_of_square(n, r)) < 1e-13
    # a pure state has Tr(rho^2) = 1
    v = np.random.default_rng(4).standard_normal(1 << 9) + 0j
    v /= np.linalg.norm(v)
    pure = _dm(engine, np.outer(v, v.conj()))
    assert abs(pure.trace_of_square() - 1.0) < 1e-13


def test_complex64_storage(engine, port):
    rho = _rho(7, 11)
    d = _dm(engine, rho, engine.KT_C64)
    got = d.partial_trace([6, 2]).download()
    np.testing.assert_allclose(got, port.dm_partial_trace(7, rho, [6, 2]), rtol=0, atol=1e-6)
    small = _dm(engine, _rho(2, 12), engine.KT_C64)
    t = small.tensor_product(d)
    np.testing.assert_allclose(t.download(), port.dm_tensor_product(2, _rho(2, 12), 7, rho), rtol=0, atol=1e-6)
    assert abs(d.trace_of_square() - port.dm_trace_of_square(7, rho)) < 1e-6


def test_prepared_density_matrix_runs_compiled_blocks(engine, port):
    """kt_dm_prepare compiles the blocks of the 2n-bit gate stream kt_dm_apply
    plans: the next apply of that circuit launches them (jit_stats) and gives
    the unprepared result (1e-12) and the oracle's rho (1e-12)."""
    from conftest import basis
    from kettle_b200 import workloads as W
    n = 7
    gates = W.random_layers(n, 6, seed=31, mixed=True)
    plain = capi.DensityMatrix(n)
    plain.apply(gates)
    want = plain.download()
    plain.close()
    dm = capi.DensityMatrix(n)
    dm.prepare(gates)
    before = capi.jit_stats()
    dm.apply(gates)
    after = capi.jit_stats()
    got = dm.download()
    dm.close()
    assert not after["failed"] and after["launches"] > before["launches"]
    assert np.abs(got - want).max() < 1e-12
    psi = port.apply(n, basis(n), gates)
    assert np.abs(got - np.outer(psi, psi.conj())).max() < 1e-12
