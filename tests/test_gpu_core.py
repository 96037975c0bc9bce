"""GPU parity: the CUDA engine, called through the C-ABI, against the oracle.

Tolerances: complex128 amplitudes and expectation values within 1e-12
(absolute, states are normalised); pair indices and sampled outcomes
bit-exact; complex64 results are reported against the complex128 oracle with
a loose bound (1e-4) since the bulk storage is single precision.
"""
import math

import numpy as np
import pytest

from conftest import basis, random_state
from kettle_b200 import capi
from kettle_b200 import workloads as W
from kettle_b200.capi import KT_APPLY_FUSED, KT_APPLY_PER_GATE, KT_C64, KT_C128, OP

pytestmark = pytest.mark.gpu

TOL = 1e-12
ALL_OPS = [g for g in capi.GATES if g != "M"]


def _gate_for(name, t, c, rng):
    if name in ("U", "CU"):
        return W.gate(name, t, control=c, u=W.haar_unitary2(rng))
    if name in capi.ANGLE_GATES:
        return W.gate(name, t, control=c, angle=float(rng.uniform(0, 2 * math.pi)))
    return W.gate(name, t, control=c)


def _run(n, init, gates, params=None, mode=KT_APPLY_FUSED, dtype=KT_C128):
    sv = capi.Statevector(n, dtype)
    sv.upload(init)
    sv.apply(gates, params, mode)
    out = sv.download()
    sv.close()
    return out


def inverse(gates):
    """Gate list of the inverse circuit (reversed, each gate replaced by its adjoint)."""
    adj = {"S": "SDAG", "SDAG": "S", "T": "TDAG", "TDAG": "T", "SX": "SXDAG", "SXDAG": "SX",
           "CS": "CSDAG", "CSDAG": "CS", "CT": "CTDAG", "CTDAG": "CT", "CSX": "CSXDAG", "CSXDAG": "CSX"}
    out = gates[::-1].copy()
    for g in out:
        name = capi.GATES[g["op"]]
        if name in adj:
            g["op"] = OP[adj[name]]
        elif name in capi.ANGLE_GATES:
            g["angle"] = -g["angle"]
        elif name in ("U", "CU"):
            u = g["u"]
            m = np.array([[u[0] + 1j * u[1], u[2] + 1j * u[3]], [u[4] + 1j * u[5], u[6] + 1j * u[7]]]).conj().T
            g["u"][:] = [m[0, 0].real, m[0, 0].imag, m[0, 1].real, m[0, 1].imag,
                         m[1, 0].real, m[1, 0].imag, m[1, 1].real, m[1, 1].imag]
    return out


# --- pair enumeration ----------------------------------------------------------

def test_pairs_small_exhaustive(engine, port, golden):
    for n in range(1, 8):
        for t in range(n):
            assert np.array_equal(capi.pairs_single(n, t), port.pairs_single(n, t))
            for c in range(n):
                if c == t or n < 2:
                    continue
                for quad in (False, True):
                    assert np.array_equal(capi.pairs_double(n, c, t, quad), port.pairs_double(n, c, t, quad))
    for a, b in ((10, 15), (7, 10), (3, 7), (0, 5), (9, 13)):
        assert np.array_equal(capi.pairs_single(5, 3, a, b - a), golden[f"pairs_ss_5_3_{a}_{b}"])
        assert np.array_equal(capi.pairs_double(6, 2, 3, False, a, b - a), golden[f"pairs_ds_6_2_3_{a}_{b}"])


def test_pairs_large_windows(engine, port):
    rng = np.random.default_rng(7)
    for n in (20, 30, 33):
        for _ in range(4):
            t = int(rng.integers(n))
            k0 = int(rng.integers(1 << (n - 1))) // 2
            assert np.array_equal(capi.pairs_single(n, t, k0, 4096), port.pairs_single(n, t, k0, 4096))
            c = int((t + 1 + rng.integers(n - 1)) % n)
            k0 = int(rng.integers(1 << (n - 2))) // 2
            for quad in (False, True):
                assert np.array_equal(capi.pairs_double(n, c, t, quad, k0, 4096),
                                      port.pairs_double(n, c, t, quad, k0, 4096))


# --- gate sweeps -----------------------------------------------------------------

@pytest.mark.parametrize("mode", [KT_APPLY_PER_GATE, KT_APPLY_FUSED])
def test_every_gate_every_position(engine, port, mode):
    rng = np.random.default_rng(11)
    for n in (1, 2, 3, 5):
        for name in ALL_OPS:
            ctl = name in capi.CONTROLLED
            if ctl and n < 2:
                continue
            for t in range(n):
                for c in (range(n) if ctl else [0]):
                    if ctl and c == t:
                        continue
                    init = random_state(n, int(rng.integers(1 << 30)))
                    g = _gate_for(name, t, c, rng)
                    got = _run(n, init, g, mode=mode)
                    want = port.apply(n, init, g)
                    assert np.abs(got - want).max() < 1e-14, (name, n, t, c)


@pytest.mark.parametrize("n,layers,mixed", [(10, 12, False), (10, 8, True), (14, 6, True), (17, 4, True)])
@pytest.mark.parametrize("mode", [KT_APPLY_PER_GATE, KT_APPLY_FUSED])
def test_random_circuits_c128(engine, port, n, layers, mixed, mode):
    g = W.random_layers(n, layers, seed=100 + n, mixed=mixed)
    init = basis(n)
    got = _run(n, init, g, mode=mode)
    want = port.apply(n, init, g)
    assert np.abs(got - want).max() < TOL


def test_golden_circuits(engine, golden):
    for key in golden:
        if key.startswith("circ_") and key.endswith("_gates"):
            stem = key[: -len("_gates")]
            n = int(stem.split("_")[1])
            got = _run(n, basis(n), golden[key])
            assert np.abs(got - golden[stem + "_amps"]).max() < TOL, stem


def test_parameterised_circuit(engine, port, golden):
    g, p = golden["hea_5_3_gates"], golden["hea_5_3_params"]
    got = _run(5, basis(5), g, p)
    assert np.abs(got - golden["hea_5_3_amps"]).max() < TOL
    g2, p2 = W.hea(12, 4, seed=3)
    assert np.abs(_run(12, basis(12), g2, p2) - port.apply(12, basis(12), g2, p2)).max() < TOL


def test_complex64_against_c128_oracle(engine, port):
    n = 14
    g = W.random_layers(n, 6, seed=5, mixed=True)
    got = _run(n, basis(n), g, dtype=KT_C64)
    want = port.apply(n, basis(n), g)
    err = np.abs(got - want).max()
    assert err < 1e-4, err


def test_inverse_circuit_returns_to_start(engine):
    n = 22
    g = W.random_layers(n, 6, seed=9, mixed=True)
    both = np.concatenate([g, inverse(g)])
    sv = capi.Statevector(n)
    sv.apply(both)
    amps = sv.download()
    assert abs(amps[0] - 1.0) < 1e-11
    assert np.abs(amps[1:]).max() < 1e-11


def test_fused_matches_per_gate_large(engine):
    n = 26
    g = W.random_layers(n, 3, seed=21, mixed=True)
    a = capi.Statevector(n)
    b = capi.Statevector(n)
    a.apply(g, mode=KT_APPLY_FUSED)
    b.apply(g, mode=KT_APPLY_PER_GATE)
    x, y = a.download(), b.download()
    assert np.abs(x - y).max() < TOL
    assert abs(a.norm_sq() - 1.0) < 1e-11


def test_bad_gates_rejected(engine):
    sv = capi.Statevector(4)
    with pytest.raises(capi.KettleError):
        sv.apply(W.gate("H", 4))
    with pytest.raises(capi.KettleError):
        sv.apply(W.gate("CX", 1, control=1))
    with pytest.raises(capi.KettleError):
        sv.apply(W.gate("M", 0))
    with pytest.raises(capi.KettleError):
        sv.apply(W.gate("RX", 0, param=3), params=np.zeros(2))
    # the state is untouched and still usable
    assert abs(sv.download()[0] - 1) == 0


# --- expectation values -------------------------------------------------------------

def test_expectation_random(engine, port):
    for n, seed in ((6, 1), (12, 2), (16, 3)):
        psi = port.apply(n, basis(n), W.random_layers(n, 4, seed=seed, mixed=True))
        strs, cs = W.random_paulis(n, 60, seed)
        sv = capi.Statevector(n)
        sv.upload(psi)
        terms, total = sv.expect(strs, cs)
        want_t, want = port.expect(n, psi, strs, cs)
        assert np.abs(terms - want_t).max() < TOL
        assert abs(total - want) < TOL * 10


def test_expectation_kats(engine, kats):
    for case in kats["expect"]:
        n = case["n"]
        strs, cs = [], []
        for (cr, ci), terms in case["ops"]:
            strs.append(W.pauli(n, {int(k): v for k, v in terms.items()}))
            cs.append(complex(cr, ci))
        sv = capi.Statevector(n)
        sv.upload(np.array([complex(a, b) for a, b in case["state"]]))
        _, total = sv.expect(np.concatenate(strs), np.array(cs))
        assert abs(total - complex(*case["expected"])) < 1e-14, case["cite"]


def test_expectation_phases_and_shared_masks(engine, port):
    n = 9
    psi = random_state(n, 4)
    strs = np.concatenate([W.pauli(n, {0: "X", 3: "Y"}, phase=ph) for ph in range(4)] +
                          [W.pauli(n, {0: "X", 3: "X", 5: "Z"}), W.pauli(n, {0: "Y", 3: "Y"}),
                           W.pauli(n, {}), W.pauli(n, {8: "Z", 2: "Z"})])
    sv = capi.Statevector(n)
    sv.upload(psi)
    t, _ = sv.expect(strs)
    want, _ = port.expect(n, psi, strs)
    assert np.abs(t - want).max() < TOL


def test_expectation_c64(engine, port):
    n = 12
    psi = port.apply(n, basis(n), W.random_layers(n, 4, seed=8, mixed=True))
    strs, cs = W.random_paulis(n, 40, 8)
    sv = capi.Statevector(n, KT_C64)
    sv.upload(psi)
    _, total = sv.expect(strs, cs)
    _, want = port.expect(n, psi, strs, cs)
    assert abs(total - want) < 1e-5


# --- probabilities, sampling, M ------------------------------------------------------------

def test_probabilities_bit_exact(engine, port, golden):
    a = golden["circ_6_8_0_11_amps"]
    sv = capi.Statevector(6)
    sv.upload(a)
    assert np.array_equal(sv.probabilities(), port.probabilities(6, a))
    assert np.array_equal(sv.probabilities(golden["noise_vec"]), golden["noise_probs"])


def test_sampling_bit_exact_golden(engine, port, golden):
    for key in golden:
        if key.startswith("circ_") and key.endswith("_amps"):
            stem = key[: -len("_amps")]
            n = int(stem.split("_")[1])
            sv = capi.Statevector(n)
            sv.upload(golden[key])
            for seed in (1, 42):
                for mode in (0, 1):
                    idx, _ = sv.sample(port.canonicals(seed, 512), mode=mode)
                    assert np.array_equal(idx, golden[f"{stem}_samples_{seed}"]), (stem, seed, mode)


def test_sampling_bit_exact_random(engine, port):
    for n, seed in ((12, 1), (18, 2), (20, 3)):
        psi = port.apply(n, basis(n), W.random_layers(n, 6, seed=seed))
        sv = capi.Statevector(n)
        sv.upload(psi)
        can = port.canonicals(seed, 4096)
        idx, rescanned = sv.sample(can)
        want = port.sample(n, port.probabilities(n, psi), can)
        assert np.array_equal(idx, want)
        noise = np.linspace(0, 0.1, n)
        idx2, _ = sv.sample(can, noise=noise)
        assert np.array_equal(idx2, port.sample(n, port.probabilities(n, psi, noise), can))


def test_sampling_edge_cases(engine, port):
    for vec in ([0.6, 0.8, 0, 0], [0, 1.0, 0, 0, 0, 0, 0, 0], [1.0, 0, 0, 0], [0, 0, 0, 1.0]):
        v = np.array(vec, dtype=np.complex128)
        n = int(np.log2(v.size))
        sv = capi.Statevector(n)
        sv.upload(v)
        can = np.concatenate([port.canonicals(3, 64), [0.0, np.nextafter(1.0, 0.0)]])
        for mode in (0, 1):
            idx, _ = sv.sample(can, mode=mode)
            assert np.array_equal(idx, port.sample(n, port.probabilities(n, v), can)), (vec, mode)


def test_measure_gate(engine, port, golden):
    a0 = golden["meas_pre_amps"]
    for (seed, q), o, a1 in zip(golden["meas_seed_qubit"], golden["meas_outcome"], golden["meas_amps"]):
        sv = capi.Statevector(5)
        sv.upload(a0)
        p0, p1 = sv.measure_probs(int(q))
        _, _, wp0, wp1 = port.measure(5, a0, int(q), 0.5)
        assert abs(p0 - wp0) < 1e-14 and abs(p1 - wp1) < 1e-14
        c0 = port.canonicals(int(seed), 1)[0]
        outcome = 0 if c0 <= p0 / (p0 + p1) else 1
        assert outcome == o
        sv.collapse(int(q), outcome, math.sqrt(1.0 / (p0 if outcome == 0 else p1)))
        assert np.abs(sv.download() - a1).max() < 1e-14


def test_norm_and_inner(engine):
    n = 10
    x, y = random_state(n, 1), random_state(n, 2)
    a, b = capi.Statevector(n), capi.Statevector(n)
    a.upload(x)
    b.upload(y)
    assert abs(a.norm_sq() - 1.0) < 1e-14
    assert abs(a.inner(b) - np.vdot(x, y)) < 1e-14


# --- density matrix -----------------------------------------------------------------------

@pytest.mark.parametrize("n,layers", [(3, 3), (4, 2), (6, 3)])
@pytest.mark.parametrize("mode", [KT_APPLY_PER_GATE, KT_APPLY_FUSED])
def test_density_matrix(engine, port, n, layers, mode):
    g = W.random_layers(n, layers, seed=40 + n, mixed=True)
    dm = capi.DensityMatrix(n)
    dm.apply(g, mode=mode)
    got = dm.download()
    rho0 = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    rho0[0, 0] = 1
    want = port.simulate_dm(n, rho0, g)
    assert np.abs(got - want).max() < TOL
    strs, cs = W.random_paulis(n, 30, n)
    t, total = dm.expect(strs, cs)
    wt, wtotal = port.dm_expect(n, want, strs, cs)
    assert np.abs(t - wt).max() < TOL and abs(total - wtotal) < TOL
    # pure-state identity: Tr(P |psi><psi|) = <psi|P|psi>
    psi = port.apply(n, basis(n), g)
    st, _ = port.expect(n, psi, strs, cs)
    assert np.abs(t - st).max() < TOL
    assert abs(dm.trace() - 1.0) < TOL


def test_density_matrix_golden(engine, golden):
    for key in golden:
        if key.startswith("dm_") and key.endswith("_gates"):
            stem = key[: -len("_gates")]
            n = int(stem.split("_")[1])
            dm = capi.DensityMatrix(n)
            dm.apply(golden[key])
            assert np.abs(dm.download() - golden[stem + "_rho"]).max() < TOL


def test_sampling_exact_tier_adversarial(engine, port):
    """The exact scan (mode 1, and every N above 2^22) against std::partial_sum
    semantics on vectors with exact ties, zeros, tiny and dyadic values."""
    rng = np.random.default_rng(17)
    cases = []
    v = np.zeros(1 << 12, dtype=np.complex128)
    v[::3] = 2.0 ** -rng.integers(3, 40, size=v[::3].size)        # dyadic: exact ties in many binades
    cases.append(v)
    w = (rng.standard_normal(1 << 13) * 1e-160).astype(np.complex128)  # tiny running sums first
    w[5000:] = rng.standard_normal((1 << 13) - 5000)
    cases.append(w)
    z = np.zeros(1 << 11, dtype=np.complex128)
    z[700] = 1.0
    z[701:710] = 2.0 ** -30
    cases.append(z)
    cases.append(random_state(14, 3))
    for vec in cases:
        n = int(np.log2(vec.size))
        sv = capi.Statevector(n)
        sv.upload(vec)
        can = np.concatenate([port.canonicals(5, 2000), [0.0, np.nextafter(1.0, 0.0)]])
        idx, rescanned = sv.sample(can, mode=1)
        assert rescanned == 1
        assert np.array_equal(idx, port.sample(n, port.probabilities(n, vec), can))


def test_sampling_large_state_exact(engine, port):
    n = 24
    psi = random_state(n, 21)
    sv = capi.Statevector(n)
    sv.upload(psi)
    can = port.canonicals(77, 4096)
    idx, rescanned = sv.sample(can)
    assert rescanned == 1  # above 2^22 amplitudes the exact scan runs directly
    assert np.array_equal(idx, port.sample(n, port.probabilities(n, psi), can))


@pytest.mark.parametrize("n,mode", [(18, 1), (23, 0)])
def test_sampling_complex64_state(engine, port, n, mode):
    """A complex64 state's shots: |a_i|^2 is formed from the FP32 amplitudes
    widened to FP64, so the oracle's sequential CDF over the stored values
    (downloaded, exact in complex128) gives the same indices, also for
    draws placed on tile boundaries."""
    sv = capi.Statevector(n, capi.KT_C64)
    sv.upload(random_state(n, 40 + n))
    stored = sv.download()
    probs = port.probabilities(n, stored)
    rng = np.random.default_rng(n)
    tiles = np.arange(0, 1 << n, 16384)
    pos = np.unique(np.clip(np.concatenate([tiles - 1, tiles, rng.integers(0, 1 << n, 500)]), 0, (1 << n) - 1))
    can = np.concatenate([_exact_probes(probs, pos[:: max(1, pos.size // 1500)]), port.canonicals(13, 2000)])
    idx, rescanned = sv.sample(can, mode=mode)
    assert rescanned == 1
    assert np.array_equal(idx, port.sample(n, probs, can))
    sv.close()


def _exact_probes(probs, positions):
    """Canonicals c whose drawn value u = c * bound lands exactly on the
    sequential CDF value at `positions` or one ulp above it: a device CDF that
    differs by one ulp at such an element changes the sampled index."""
    cdf = np.cumsum(probs)  # sequential left-to-right, as std::partial_sum
    last = cdf[-1]
    below = cdf[cdf < last]
    second = below[-1] if below.size else 0.0
    bound = last - (last - second) * 1.0e-4
    out = []
    for i in positions:
        for target in (cdf[i], np.nextafter(cdf[i], np.inf)):
            if not (0.0 < target <= bound):
                continue
            c = target / bound
            for cc in (c, np.nextafter(c, 0.0), np.nextafter(c, 1.0)):
                if 0.0 <= cc < 1.0 and cc * bound + 0.0 == target:
                    out.append(cc)
                    break
    return np.array(out)


@pytest.mark.parametrize("case", ["random", "zero_prefix", "dyadic", "dominant", "uniform", "tiny_head"])
def test_sampling_exact_tier_probes(engine, port, case):
    """The tiled exact CDF (several 16384-element tiles) probed at tile
    boundaries and random elements, against std::partial_sum semantics."""
    n = 18
    N = 1 << n
    rng = np.random.default_rng(sum(map(ord, case)))
    if case == "random":
        v = random_state(n, 5)
    elif case == "zero_prefix":
        v = np.zeros(N, dtype=np.complex128)
        v[40000:] = rng.standard_normal(N - 40000)
    elif case == "dyadic":
        v = np.zeros(N, dtype=np.complex128)
        v[::3] = 2.0 ** (-rng.integers(3, 30, size=v[::3].size) / 2.0)
    elif case == "dominant":
        v = (rng.standard_normal(N) * 1e-4).astype(np.complex128)
        v[100000] = 1.0
    elif case == "uniform":
        v = np.full(N, 2.0 ** (-n / 2), dtype=np.complex128)
    else:
        v = rng.standard_normal(N).astype(np.complex128)
        v[:30000] *= 1e-170
    sv = capi.Statevector(n)
    sv.upload(v)
    probs = port.probabilities(n, v)
    tiles = np.arange(0, N, 16384)
    pos = np.unique(np.clip(np.concatenate([tiles - 1, tiles, tiles + 1, rng.integers(0, N, 3000)]), 0, N - 1))
    can = np.concatenate([_exact_probes(probs, pos), port.canonicals(9, 2000)])
    assert can.size > 2000
    idx, rescanned = sv.sample(can, mode=1)
    assert rescanned == 1
    assert np.array_equal(idx, port.sample(n, probs, can))


def _perm_heavy(n, layers, seed):
    """Layers of X / CX / CCX-free permutation gates mixed with rotations and
    diagonal gates, with controls and targets spread over every qubit."""
    rng = np.random.default_rng(seed)
    recs = []
    for _ in range(layers):
        for q in range(n):
            r = rng.integers(6)
            if r == 0:
                recs.append(W.gate("X", q))
            elif r == 1:
                recs.append(W.gate("RY", q, angle=float(rng.uniform(0, 6.28))))
            elif r == 2:
                recs.append(W.gate("RZ", q, angle=float(rng.uniform(0, 6.28))))
            elif r == 3:
                recs.append(W.gate("H", q))
        for _ in range(n):
            c, t = rng.choice(n, 2, replace=False)
            recs.append(W.gate("CX", int(t), control=int(c)))
        c, t = rng.choice(n, 2, replace=False)
        recs.append(W.gate("CRX", int(t), control=int(c), angle=0.7))
        recs.append(W.gate("CZ", int(t), control=int(c)))
    return np.concatenate(recs)


@pytest.mark.parametrize("n", [10, 14, 20])
def test_permutation_folding(engine, port, n):
    """X / CX folded into the transposes give the oracle's state, and the
    same state as running them as ops (knob off) and as per-gate sweeps."""
    g = _perm_heavy(n, 6, seed=n)
    want = port.apply(n, basis(n), g)
    old = capi.tuning_get("fold_permutations")
    try:
        states = []
        for f in (1, 0):
            capi.tuning_set("fold_permutations", f)
            sv = capi.Statevector(n)
            sv.apply(g)
            states.append(sv.download())
            sv.close()
    finally:
        capi.tuning_set("fold_permutations", old)
    assert np.abs(states[0] - want).max() < TOL
    assert np.abs(states[1] - want).max() < TOL
    assert np.abs(states[0] - states[1]).max() < 1e-13
    # complex64 with folding
    sv = capi.Statevector(n, capi.KT_C64)
    sv.apply(g)
    assert np.abs(sv.download() - want).max() < 1e-4


def test_statevector_tensor_product_and_diagonal_expectation(engine, port):
    """kt_sv_tensor_product (state/state.cpp:144-157: left qubits low) and
    kt_sv_diagonal_expectation (state/state.cpp:174-188) against numpy."""
    nl, nr = 7, 6
    a = random_state(nl, 1)
    b = random_state(nr, 2)
    L = capi.Statevector(nl)
    R = capi.Statevector(nr)
    L.upload(a)
    R.upload(b)
    out = L.tensor_product(R)
    want = np.kron(b, a)  # index i_l + i_r 2^nl
    assert np.abs(out.download() - want).max() < 1e-15
    lam = np.random.default_rng(3).standard_normal(1 << (nl + nr)) + 1j * np.random.default_rng(4).standard_normal(1 << (nl + nr))
    got = out.diagonal_expectation(lam)
    assert abs(got - np.sum(np.conj(want) * lam * want)) < 1e-12
    for h in (L, R, out):
        h.close()


def test_sampling_from_a_probability_vector(engine, port):
    """kt_sample_probabilities: the sampler of kt_sv_sample on a caller's vector,
    bit-exact with the oracle's sequential CDF and lower_bound, also for a
    length that is not a power of two."""
    rng = np.random.default_rng(9)
    for size in (3, 1000, 1 << 14):
        p = rng.random(size) ** 3
        p /= p.sum()
        can = port.canonicals(11, 2048)
        got = capi.sample_probabilities(p, can)
        assert np.array_equal(got, port.sample_raw(p, can)), size


def test_density_matrix_measurement(engine, port):
    """M on a density matrix (measure_density_matrix.cpp:22-105): P(b) is the
    sum of |rho(r, c)|^2 over rows and columns with bit b; the outcome's block
    is kept and scaled, the other three cleared."""
    n = 5
    g = W.random_layers(n, 3, seed=12, mixed=True)
    dm = capi.DensityMatrix(n)
    dm.apply(g)
    rho = dm.download()
    for q in range(n):
        bits = (np.arange(1 << n) >> q) & 1
        same0 = np.outer(bits == 0, bits == 0)
        same1 = np.outer(bits == 1, bits == 1)
        p0, p1 = dm.measure_probs(q)
        assert abs(p0 - np.sum(np.abs(rho[same0]) ** 2)) < 1e-13
        assert abs(p1 - np.sum(np.abs(rho[same1]) ** 2)) < 1e-13
    q, o = 2, 1
    p0, p1 = dm.measure_probs(q)
    s = np.sqrt(1.0 / p1)
    dm.collapse(q, o, s)
    bits = (np.arange(1 << n) >> q) & 1
    want = np.where(np.outer(bits == o, bits == o), rho * s, 0.0)
    assert np.abs(dm.download() - want).max() < 1e-14
    dm.close()
