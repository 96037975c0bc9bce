"""The dense five-qubit block on the tensor cores (kt_sv_apply_dense5).

A random 32 x 32 unitary on qubits 0..4 of a complex64 state, applied as a
tcgen05 GEMM, against the complex128 product on the host:
  * passes = 3 and 4 (operands split into TF32 parts, three or four
    products): within 5e-6 of the largest amplitude, and within 8x the
    error of an FP32 GEMM on the host (numpy complex64 matmul) on the same
    data (measured about 5x: the tensor cores' FP32 accumulation, not the
    operand split, sets it, as four products are no better than three);
  * passes = 1 (one plain TF32 product): coarser, within 5e-3, and at least
    10x the error of passes = 3;
at sizes of one CTA tile (12 qubits) up to more tiles than SMs, plus U then
U^dagger at 24 qubits back to the input, and the argument checks.
"""
import numpy as np
import pytest

from kettle_b200 import capi

pytestmark = pytest.mark.gpu


def _unitary(seed):
    rng = np.random.default_rng(seed)
    z = (rng.normal(size=(32, 32)) + 1j * rng.normal(size=(32, 32))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def _state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return (v / np.linalg.norm(v)).astype(np.complex64)


def _apply(n, x, u, passes):
    sv = capi.Statevector(n, capi.KT_C64)
    sv.upload(x)
    sv.apply_dense5(u, passes=passes)
    out = sv.download()
    sv.close()
    return out


@pytest.mark.parametrize("n", [12, 13, 17, 20])
def test_dense5_matches_host_product(engine, n):
    u = _unitary(n)
    x = _state(n, 100 + n)
    # every row of 32 consecutive amplitudes is mapped by U: y_b = sum_a U[b][a] x_a
    want = (x.astype(np.complex128).reshape(-1, 32) @ u.T).reshape(-1)
    f32 = (x.reshape(-1, 32) @ u.astype(np.complex64).T).reshape(-1)
    scale = np.abs(want).max()
    e_f32 = np.abs(f32 - want).max() / scale
    e4 = np.abs(_apply(n, x, u, 4) - want).max() / scale
    e3 = np.abs(_apply(n, x, u, 3) - want).max() / scale
    e1 = np.abs(_apply(n, x, u, 1) - want).max() / scale
    print(f"n={n}: relative max error fp32 {e_f32:.3g}, 4 products {e4:.3g}, 3 products {e3:.3g}, tf32 {e1:.3g}")
    assert e4 < 5e-6 and e4 < 8 * e_f32 + 1e-7, (e4, e_f32)
    assert e3 < 5e-6 and e3 < 8 * e_f32 + 1e-7, (e3, e_f32)
    assert e1 < 5e-3 and e1 > 10 * e3, (e1, e3)


def test_dense5_round_trip_at_24_qubits(engine):
    n = 24
    u = _unitary(7)
    x = _state(n, 8)
    sv = capi.Statevector(n, capi.KT_C64)
    sv.upload(x)
    sv.apply_dense5(u)
    mid = sv.download()
    sv.apply_dense5(u.conj().T)
    back = sv.download()
    sv.close()
    assert abs(np.linalg.norm(mid) - 1.0) < 1e-5
    assert np.abs(mid - x).max() > 1e-3  # U did act
    assert np.abs(back - x).max() < 1e-5 * np.abs(x).max() * 32


def test_dense5_argument_checks(engine):
    u = _unitary(1)
    sv = capi.Statevector(12)  # complex128
    with pytest.raises(capi.KettleError):
        sv.apply_dense5(u)
    sv.close()
    sv = capi.Statevector(11, capi.KT_C64)
    with pytest.raises(capi.KettleError):
        sv.apply_dense5(u)
    sv.close()
    sv = capi.Statevector(12, capi.KT_C64)
    with pytest.raises(capi.KettleError):
        sv.apply_dense5(u, passes=2)
    sv.close()
