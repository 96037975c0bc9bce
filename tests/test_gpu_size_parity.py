"""Parity at the benchmark configurations' own sizes, against sources
independent of the engine:

* config 1 in full (20 qubits, 100 layers, all 200 strings, 4096 shots)
  against the reference library's own outputs (tests/golden/golden_size.npz,
  made by tests/golden/make_golden.py from the compiled reference);
* the 13-qubit density matrix of config 2b (2^26 entries, 26 index bits, so
  run-time compiled blocks too) against |psi><psi| with psi from the oracle,
  and Tr(P rho) of its 200 strings against the oracle's <psi|P|psi>;
* product states at 30 qubits complex128 and 33 qubits complex64 (above 2^31
  amplitudes): the benchmark gate family on two or three disjoint, interleaved
  registers of <= 15 qubits, run through compiled blocks whose tiles mix the
  registers; amplitudes at thousands of indices against the Kronecker product
  of the oracle's register states, and Pauli expectations (which read every
  amplitude) against products of the registers' values;
* the 30-qubit benchmark circuit followed by its inverse returns to |0...0>;
* the 24-qubit, 384-parameter adjoint gradient against central finite
  differences (h = 1e-5) of complex128 forward passes.
"""
import numpy as np
import pytest

from conftest import GOLDEN, basis
from kettle_b200 import capi
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12


class _DeviceArray:
    """A raw device buffer seen by torch (__cuda_array_interface__)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}


def gather(sv, index):
    """Amplitudes of a device statevector at `index`, gathered on the device."""
    import torch
    n_amps = 1 << sv.n_qubits
    if sv.dtype == capi.KT_C128:
        raw = torch.as_tensor(_DeviceArray(sv.device_ptr(), 2 * n_amps, "<f8"), device="cuda")
    else:
        raw = torch.as_tensor(_DeviceArray(sv.device_ptr(), 2 * n_amps, "<f4"), device="cuda")
    torch.cuda.synchronize()
    ix = torch.as_tensor(np.asarray(index, dtype=np.int64), device="cuda")
    re = raw[2 * ix].double().cpu().numpy()
    im = raw[2 * ix + 1].double().cpu().numpy()
    return re + 1j * im


def state_sums(amps):
    """sum |a_i|^2 i and sum a_i w^(7 i), w = e^{-2 pi i / N}: the two sums
    tests/golden/make_golden.py stores beside the probe amplitudes."""
    N = amps.size
    i = np.arange(N, dtype=np.float64)
    s2 = complex(np.sum(amps * np.exp(-2j * np.pi * 7.0 * i / N)))
    return [float(np.sum(np.abs(amps) ** 2 * i)), s2.real, s2.imag]


@pytest.fixture()
def jit_mode(engine):
    old = capi.tuning_get("fused_jit")
    yield capi
    capi.tuning_set("fused_jit", old)


# ---------------------------------------------------------------- config 1 ----
@pytest.mark.parametrize("fused_jit", [2, 1])
def test_config1_full_against_reference(jit_mode, fused_jit):
    """20 q, 100 layers (2950 gates), <P_k> of 200 strings, 4096 shots: the
    reference library's own values (simulate.cpp:265-597,
    pauli_operator.cpp:76-103, measurements.cpp:235-311).  fused_jit 2 is the
    default path (precompiled fused blocks at 20 q), 1 the compiled blocks."""
    capi.tuning_set("fused_jit", fused_jit)
    g = dict(np.load(GOLDEN / "golden_size.npz"))
    n = 20
    sv = capi.Statevector(n)
    sv.apply(g["c1_gates"])
    amps = sv.download()
    assert np.abs(amps[g["c1_probe_index"]] - g["c1_probe_amps"]).max() < TOL
    s = state_sums(amps)
    assert abs(s[0] - g["c1_sums"][0]) < 1e-12 * (1 << n)
    assert abs(complex(s[1], s[2]) - complex(g["c1_sums"][1], g["c1_sums"][2])) < 1e-10
    terms, total = sv.expect(g["c1_strings"], g["c1_coeffs"])
    assert np.abs(terms - g["c1_terms"]).max() < TOL
    assert abs(total - g["c1_total"][0]) < TOL
    idx, _ = sv.sample(capi.canonicals_mt19937(2024, 4096))
    assert np.array_equal(idx, g["c1_samples"])
    sv.close()


# --------------------------------------------------------------- config 2b ----
@pytest.mark.parametrize("fused_jit", [2, 1])
def test_config2b_density_matrix_13q(jit_mode, port, fused_jit):
    """13-qubit density matrix, the 100-layer config-1 circuit family: rho must
    be |psi><psi| (the reference's own cross-check,
    simulate_density_matrix_test.cpp:24-150) with psi from the oracle, and
    Tr(P rho) = <psi|P|psi> for the 200 strings."""
    capi.tuning_set("fused_jit", fused_jit)
    n = 13
    gates = W.random_layers(n, 100, seed=2024, mixed=False)
    strings, coeffs = W.random_paulis(n, 200, seed=2024)
    psi = port.apply(n, basis(n), gates)
    dm = capi.DensityMatrix(n)
    dm.set_basis(0)
    dm.apply(gates)
    if fused_jit == 1:
        assert capi.jit_stats()["launches"] > 0
    rho = dm.download()
    N = 1 << n
    worst = 0.0
    for c0 in range(0, N, 512):
        blk = np.outer(psi, psi[c0:c0 + 512].conj())
        worst = max(worst, float(np.abs(rho[:, c0:c0 + 512] - blk).max()))
    assert worst < TOL, worst
    del rho
    terms, total = dm.expect(strings, coeffs)
    want_terms, want_total = port.expect(n, psi, strings, coeffs)
    assert np.abs(terms - want_terms).max() < TOL
    assert abs(total - want_total) < TOL
    assert abs(dm.trace() - 1.0) < TOL
    dm.close()


# ------------------------------------------------------- product structure ----
def _register_circuit(n_total, regs, layers, seed):
    """The benchmark gate family run independently on each register (a list of
    physical qubit lists), interleaved 10 gates at a time; returns the gate
    list and each register's own circuit."""
    local = [W.random_layers(len(r), layers, seed=seed + k, mixed=True) for k, r in enumerate(regs)]
    mapped = []
    for r, g in zip(regs, local):
        m = g.copy()
        m["target"] = np.asarray(r, dtype=np.uint32)[g["target"]]
        m["control"] = np.asarray(r, dtype=np.uint32)[g["control"]]
        mapped.append(m)
    out, pos = [], [0] * len(mapped)
    while any(p < m.size for p, m in zip(pos, mapped)):
        for k, m in enumerate(mapped):
            out.append(m[pos[k]:pos[k] + 10])
            pos[k] += 10
    return np.concatenate(out), local


def _split_index(index, regs):
    """Global indices -> each register's local index."""
    out = []
    for r in regs:
        loc = np.zeros_like(index)
        for j, q in enumerate(r):
            loc |= ((index >> q) & 1) << j
        out.append(loc)
    return out


def _product_strings(regs, count, seed):
    """Random Pauli strings over all registers, and each register's part."""
    n = sum(len(r) for r in regs)
    strings, _ = W.random_paulis(n, count, seed=seed)
    parts = []
    for r in regs:
        p = np.zeros(count, dtype=capi.PAULI_DTYPE)
        for j, q in enumerate(r):
            p["x"] |= ((strings["x"] >> np.uint64(q)) & np.uint64(1)) << np.uint64(j)
            p["z"] |= ((strings["z"] >> np.uint64(q)) & np.uint64(1)) << np.uint64(j)
        parts.append(p)
    return strings, parts


@pytest.mark.parametrize("n,dtype,n_regs", [(30, capi.KT_C128, 2), (33, capi.KT_C64, 3)])
def test_product_state_at_size(jit_mode, port, n, dtype, n_regs):
    """Compiled blocks at 30 q complex128 (16 GiB) and 33 q complex64 (64 GiB,
    2^33 amplitudes): amplitudes at 8192 indices (half of them above 2^(n-1))
    equal the Kronecker product of the registers' oracle states, and <P> of 40
    strings equals the product of the registers' <P_r>."""
    regs = [list(range(k, n, n_regs)) for k in range(n_regs)]
    gates, local = _register_circuit(n, regs, layers=12, seed=300 + n)
    psis = [port.apply(len(r), basis(len(r)), g) for r, g in zip(regs, local)]
    sv = capi.Statevector(n, dtype)
    sv.set_basis(0)
    sv.prepare(gates)
    k0 = capi.jit_stats()["launches"]
    sv.apply(gates)
    assert capi.jit_stats()["launches"] > k0, "the compiled block kernels did not run"
    rng = np.random.default_rng(n)
    index = np.concatenate([rng.integers(0, 1 << (n - 1), 4096), rng.integers(1 << (n - 1), 1 << n, 4096)])
    index = index.astype(np.int64)
    got = gather(sv, index)
    want = np.ones(index.size, dtype=np.complex128)
    for psi, loc in zip(psis, _split_index(index, regs)):
        want = want * psi[loc]
    scale = float(np.abs(want).max())
    rel = float(np.abs(got - want).max()) / scale
    if dtype == capi.KT_C128:
        assert rel < 1e-10 and float(np.abs(got - want).max()) < TOL, rel
    else:
        assert rel < 1e-4, rel
    strings, parts = _product_strings(regs, 40, seed=n)
    terms, _ = sv.expect(strings)
    prod = np.ones(strings.size, dtype=np.complex128)
    for r, psi, p in zip(regs, psis, parts):
        t, _ = port.expect(len(r), psi, p)
        prod = prod * t
    tol = TOL if dtype == capi.KT_C128 else 1e-5
    assert np.abs(terms - prod).max() < tol
    assert abs(sv.norm_sq() - 1.0) < (1e-12 if dtype == capi.KT_C128 else 1e-6)
    sv.close()


def _inverse(gates):
    """The gate list undoing `gates`: reversed, each gate replaced by its inverse."""
    inv = gates[::-1].copy()
    for k in range(inv.size):
        name = capi.GATES[int(inv["op"][k])]
        if name in capi.ANGLE_GATES:
            inv["angle"][k] = -inv["angle"][k]
        elif name == "U":
            u = inv["u"][k]
            m = np.array([[u[0] + 1j * u[1], u[2] + 1j * u[3]], [u[4] + 1j * u[5], u[6] + 1j * u[7]]])
            d = m.conj().T
            inv["u"][k] = [d[0, 0].real, d[0, 0].imag, d[0, 1].real, d[0, 1].imag,
                           d[1, 0].real, d[1, 0].imag, d[1, 1].real, d[1, 1].imag]
        else:
            assert name in ("H", "X", "CX"), name
    return inv


def test_bench_circuit_then_inverse_30q(jit_mode):
    """The 30-qubit, 40-layer benchmark circuit and then its inverse, through
    compiled blocks: the state returns to |0...0>."""
    n = 30
    gates = W.random_layers(n, 40, seed=2024, mixed=True)
    both = np.concatenate([gates, _inverse(gates)])
    sv = capi.Statevector(n)
    sv.set_basis(0)
    sv.prepare(both)
    sv.apply(both)
    a0 = gather(sv, np.array([0]))[0]
    assert abs(a0 - 1.0) < 1e-11, a0
    assert abs(sv.norm_sq() - 1.0) < 1e-11
    # every other amplitude is ~0: <Z_q> = 1 on every qubit reads them all
    zs = np.concatenate([W.pauli(n, {q: "Z"}) for q in range(n)])
    terms, _ = sv.expect(zs)
    assert np.abs(terms - 1.0).max() < 1e-11
    sv.close()


# ----------------------------------------------------------------- config 4 ----
def test_adjoint_24q_against_central_differences(engine):
    """24-qubit hardware-efficient ansatz, 384 parameters, XXZ chain with Z
    fields: the adjoint gradient against central differences (h = 1e-5) of
    complex128 forward passes, max |dg| <= 1e-8."""
    n = 24
    gates, params = W.hea(n, 8, seed=2024)
    strings, coeffs = W.xxz_chain(n, seed=2024)
    sv = capi.Statevector(n)
    sv.set_basis(0)
    adj = capi.Adjoint(sv)
    adj.forward(gates, params, strings, coeffs)
    grad = adj.backward()
    adj.close()
    h = 1e-5
    ev = capi.Statevector(n)

    def energy(p):
        ev.set_basis(0)
        ev.apply(gates, p)
        return ev.expect(strings, coeffs)[1].real

    fd = np.empty(params.size)
    for k in range(params.size):
        p = params.copy()
        p[k] += h
        ep = energy(p)
        p[k] -= 2 * h
        fd[k] = (ep - energy(p)) / (2 * h)
    assert np.abs(grad - fd).max() <= 1e-8, np.abs(grad - fd).max()
    ev.close()
    sv.close()
