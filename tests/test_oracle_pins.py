"""Pin the oracle (the C restatement in oracle/kt_oracle.c) before trusting it:
against the known-answer cases of the reference's own tests
(tests/golden/ref_kats.json), against outputs of the reference library itself
(tests/golden/golden_ref.npz) and, where the reference was compiled here
(oracle/_ref), against live runs of it on fresh seeded cases."""
import numpy as np
import pytest

from conftest import basis, random_state
from kettle_b200 import workloads as W


def _gates(items):
    out = []
    for it in items:
        name, t = it[0], it[1]
        c = it[2] if len(it) > 2 else 0
        ang = it[3] if len(it) > 3 else 0.0
        out.append(W.gate(name, t, control=c, angle=ang))
    return np.concatenate(out)


def _cx(pairs):
    return np.array([complex(a, b) for a, b in pairs], dtype=np.complex128)


def _strings(n, ops):
    strs, cs = [], []
    for (cr, ci), terms in ops:
        strs.append(W.pauli(n, {int(k): v for k, v in terms.items()}))
        cs.append(complex(cr, ci))
    return np.concatenate(strs), np.array(cs)


def apply_pauli_masks(psi, x, z):
    """P|i> = i^{#Y} (-1)^{popcount(i & z)} |i ^ x>: the closed form the device kernels use."""
    n_y = bin(x & z).count("1")
    out = np.zeros_like(psi)
    for i in range(psi.size):
        sign = -1.0 if bin(i & z).count("1") % 2 else 1.0
        out[i ^ x] += (1j ** n_y) * sign * psi[i]
    return out


# --- reference test known answers -------------------------------------------

def test_kat_statevector(port, kats):
    for case in kats["sv"]:
        n = case["n"]
        init = basis(n) if case["init"] is None else _cx(case["init"])
        got = port.apply(n, init, _gates(case["gates"]))
        np.testing.assert_allclose(got, _cx(case["expected"]), atol=1e-15, err_msg=case["name"] + " " + case["cite"])


def test_kat_pauli_apply_closed_form(kats):
    for case in kats["pauli_apply"]:
        n = case["n"]
        idx = lambda bits: sum(1 << i for i, ch in enumerate(bits) if ch == "1")  # noqa: E731
        rec = W.pauli(n, {int(k): v for k, v in case["terms"].items()})[0]
        got = apply_pauli_masks(basis(n, idx(case["init"])), int(rec["x"]), int(rec["z"]))
        want = basis(n, idx(case["out"])) * complex(*case["factor"])
        np.testing.assert_allclose(got, want, atol=0, err_msg=case["cite"])


def test_kat_expectation(port, kats):
    for case in kats["expect"]:
        n = case["n"]
        strs, cs = _strings(n, case["ops"])
        _, total = port.expect(n, _cx(case["state"]), strs, cs)
        assert abs(total - complex(*case["expected"])) < 1e-14, case["cite"]


def test_kat_cdf(port, kats):
    c = kats["cdf"]
    probs = np.array(c["probs"])
    # sampled index of u just above each CDF step (uniforms chosen on the steps)
    assert np.allclose(np.cumsum(probs), c["cdf"])
    bound = c["cdf"][-1] - (c["cdf"][-1] - c["cdf"][-2]) * 1e-4
    canon = np.array(c["cdf"]) * 0.999 / bound
    idx = port.sample(2, probs, canon)
    assert list(idx) == [0, 1, 2, 3]


# --- reference library outputs (golden vectors) -------------------------------------

def test_golden_pairs(port, golden):
    for key, want in golden.items():
        if key.startswith("pairs_s_"):
            _, _, n, t = key.split("_")
            assert np.array_equal(port.pairs_single(int(n), int(t)), want), key
        elif key.startswith("pairs_d_") or key.startswith("pairs_q_"):
            kind, n, c, t = key.split("_")[1:]
            got = port.pairs_double(int(n), int(c), int(t), quad=(kind == "q"))
            assert np.array_equal(got, want), key
        elif key.startswith("pairs_ss_"):
            a, b = map(int, key.split("_")[-2:])
            assert np.array_equal(port.pairs_single(5, 3, k0=a, count=b - a), want), key
        elif key.startswith("pairs_ds_"):
            a, b = map(int, key.split("_")[-2:])
            assert np.array_equal(port.pairs_double(6, 2, 3, k0=a, count=b - a), want), key


def test_golden_pair_sets_cover_each_index_once(golden):
    for key, v in golden.items():
        if key.startswith("pairs_s_"):
            n = int(key.split("_")[2])
            assert sorted(v.reshape(-1).tolist()) == list(range(1 << n)), key


def test_golden_circuits(port, golden):
    for key in golden:
        if not key.endswith("_gates") or not key.startswith("circ_"):
            continue
        stem = key[: -len("_gates")]
        n = int(stem.split("_")[1])
        g = golden[key]
        amps = port.apply(n, basis(n), g)
        assert np.array_equal(amps, golden[stem + "_amps"]), stem  # bit-exact with the reference
        terms, total = port.expect(n, amps, golden[stem + "_strings"], golden[stem + "_coeffs"])
        assert np.array_equal(terms, golden[stem + "_terms"]), stem
        assert total == golden[stem + "_total"][0], stem
        probs = port.probabilities(n, amps)
        for seed in (1, 42):
            idx = port.sample(n, probs, port.canonicals(seed, 512))
            assert np.array_equal(idx, golden[f"{stem}_samples_{seed}"]), (stem, seed)


def test_golden_parameterised(port, golden):
    amps = port.apply(5, basis(5), golden["hea_5_3_gates"], golden["hea_5_3_params"])
    assert np.array_equal(amps, golden["hea_5_3_amps"])


def test_golden_measure(port, golden):
    a0 = golden["meas_pre_amps"]
    for (seed, q), o, a1 in zip(golden["meas_seed_qubit"], golden["meas_outcome"], golden["meas_amps"]):
        c0 = port.canonicals(int(seed), 1)[0]
        got, outcome, _, _ = port.measure(5, a0, int(q), c0)
        assert outcome == o
        assert np.array_equal(got, a1)


def test_golden_density_matrix(port, golden):
    for key in golden:
        if key.startswith("dm_") and key.endswith("_gates"):
            stem = key[: -len("_gates")]
            n = int(stem.split("_")[1])
            rho0 = np.zeros((1 << n, 1 << n), dtype=np.complex128)
            rho0[0, 0] = 1.0
            got = port.simulate_dm(n, rho0, golden[key])
            np.testing.assert_allclose(got, golden[stem + "_rho"], atol=1e-14)


def test_golden_noise(port, golden):
    got = port.probabilities(6, golden["circ_6_8_0_11_amps"], golden["noise_vec"])
    assert np.array_equal(got, golden["noise_probs"])


def test_canonicals_restatement_matches_library_helper():
    # host-only C-ABI helper (no GPU needed): std::mt19937 + generate_canonical
    from kettle_b200 import capi
    from oracle.oracle import port as _p
    for seed in (0, 1, 42, 2**31 - 1, 12345678):
        assert np.array_equal(capi.canonicals_mt19937(seed, 1000), _p().canonicals(seed, 1000))


# --- live reference (where compiled here) ----------------------------------------

@pytest.mark.parametrize("seed", [1, 2, 3])
def test_live_reference_random(port, ref, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(3, 11))
    g = W.random_layers(n, 5, seed=seed, mixed=True)
    init = random_state(n, seed)
    a = port.apply(n, init, g)
    b, _ = ref.simulate_sv(n, init, g)
    assert np.array_equal(a, b)
    s, c = W.random_paulis(n, 20, seed + 7)
    ta, sa = port.expect(n, a, s, c)
    tb, sb = ref.expect(n, b, s, c)
    assert np.array_equal(ta, tb) and sa == sb
    noise = rng.uniform(0, 0.3, n)
    assert np.array_equal(port.probabilities(n, a, noise), ref.probabilities(n, b, noise))
    probs = port.probabilities(n, a)
    assert np.array_equal(port.sample(n, probs, port.canonicals(seed, 300)), ref.sample_memory(n, b, 300, seed))


def test_live_reference_edge_sampling(port, ref):
    # zero tail after the last non-zero probability, and a single non-zero entry
    for vec in ([0.6, 0.8, 0, 0], [0, 1.0, 0, 0, 0, 0, 0, 0], [1.0, 0, 0, 0]):
        v = np.array(vec, dtype=np.complex128)
        n = int(np.log2(v.size))
        probs = port.probabilities(n, v)
        for seed in (3, 9):
            assert np.array_equal(port.sample(n, probs, port.canonicals(seed, 64)), ref.sample_memory(n, v, 64, seed))


def test_live_reference_dm(port, ref):
    n = 3
    g = W.random_layers(n, 2, seed=5, mixed=True)
    rho0 = np.zeros((8, 8), dtype=np.complex128)
    rho0[0, 0] = 1
    np.testing.assert_allclose(port.simulate_dm(n, rho0, g), ref.simulate_dm(n, rho0, g), atol=1e-15)


# --- density-matrix operations -----------------------------------------------------

def _dm_golden():
    from conftest import GOLDEN
    return dict(np.load(GOLDEN / "golden_dm_ops.npz"))


def test_golden_partial_trace_tensor_purity(port):
    g = _dm_golden()
    sizes = sorted({int(k.split("_")[1]) for k in g if k.startswith("dmop_") and k.endswith("_rho")})
    assert sizes == [3, 4, 5]
    for n in sizes:
        rho = g[f"dmop_{n}_rho"]
        j = 0
        while f"dmop_{n}_pt_{j}_q" in g:
            got = port.dm_partial_trace(n, rho, g[f"dmop_{n}_pt_{j}_q"].tolist())
            assert np.array_equal(got, g[f"dmop_{n}_pt_{j}_out"]), (n, j)
            j += 1
        assert abs(port.dm_trace_of_square(n, rho) - g[f"dmop_{n}_tsq"][0]) < 1e-15
    got = port.dm_tensor_product(2, g["dmop_tp_left"], 3, g["dmop_tp_right"])
    assert np.array_equal(got, g["dmop_tp_out"])


def test_kat_partial_trace_of_product_states(port):
    # test/source/state/density_matrix_test.cpp:270-410: tracing one factor
    # of a tensor product out leaves the other factor
    rng = np.random.default_rng(3)
    states = []
    for _ in range(3):
        v = rng.standard_normal(2) + 1j * rng.standard_normal(2)
        v /= np.linalg.norm(v)
        states.append(np.outer(v, v.conj()))
    t01 = port.dm_tensor_product(1, states[0], 1, states[1])
    t012 = port.dm_tensor_product(2, t01, 1, states[2])
    np.testing.assert_allclose(port.dm_partial_trace(3, t012, [0]), port.dm_tensor_product(1, states[1], 1, states[2]), atol=1e-15)
    np.testing.assert_allclose(port.dm_partial_trace(3, t012, [1]), port.dm_tensor_product(1, states[0], 1, states[2]), atol=1e-15)
    np.testing.assert_allclose(port.dm_partial_trace(3, t012, [2]), t01, atol=1e-15)
    for qs, keep in (([0, 1], 2), ([1, 0], 2), ([0, 2], 1), ([2, 0], 1), ([1, 2], 0), ([2, 1], 0)):
        np.testing.assert_allclose(port.dm_partial_trace(3, t012, qs), states[keep], atol=1e-15)
    assert abs(port.dm_trace_of_square(3, t012) - 1.0) < 1e-14


def test_live_reference_dm_ops(port, ref):
    from tests.golden.make_golden import random_rho
    for n in (1, 2, 6):
        rho = random_rho(n, 40 + n)
        for qs in ([0], [n - 1], list(range(n))[::-1], [0] * (n // 2 + 1) if n > 1 else [0]):
            assert np.array_equal(port.dm_partial_trace(n, rho, qs), ref.dm_partial_trace(n, rho, qs))


# --- full-size fixtures (tests/golden/golden_size.npz) ----------------------

@pytest.fixture(scope="module")
def golden_size():
    from conftest import GOLDEN
    return dict(np.load(GOLDEN / "golden_size.npz"))


def test_golden_config1_full_size(port, golden_size):
    """The oracle on the whole 20-qubit, 100-layer benchmark configuration:
    bit-exact with the reference's final amplitudes (at the stored probes),
    <P_k> of 40 of its 200 strings and its 4096 sampled indices."""
    g = golden_size
    n = 20
    amps = port.apply(n, basis(n), g["c1_gates"])
    assert np.array_equal(amps[g["c1_probe_index"]], g["c1_probe_amps"])
    terms, _ = port.expect(n, amps, g["c1_strings"][:40], g["c1_coeffs"][:40])
    assert np.array_equal(terms, g["c1_terms"][:40])
    idx = port.sample(n, port.probabilities(n, amps), port.canonicals(2024, 4096))
    assert np.array_equal(idx, g["c1_samples"])


def test_random_unitaries_are_the_reference_generator(golden_size):
    """The benchmark circuits' U gates: generate_random_unitary2x2 on one
    std::mt19937 stream (random_u_gates.cpp:13-36), bit for bit."""
    for seed in (0, 2024):
        got = np.array(W.random_unitaries(seed, 64))
        assert np.array_equal(got, golden_size[f"ru_{seed}"]), seed


def test_random_unitaries_live_reference(ref):
    for seed in (1, 99, 123456):
        got = W.random_unitaries(seed, 40)
        want = ref.random_unitaries(seed, 40)
        assert all(np.array_equal(a, b) for a, b in zip(got, want)), seed


def test_sampling_from_probability_vectors(port, ref):
    """The oracle's sampler on any probability vector (the std::vector<double>
    overloads of perform_measurements_as_*) against the reference's own,
    including lengths that are not powers of two and zero entries."""
    rng = np.random.default_rng(5)
    for size in (1, 2, 3, 7, 100, 4096):
        p = rng.random(size) ** 2
        p[rng.random(size) < 0.2] = 0.0
        if p.sum() == 0.0:
            p[0] = 1.0
        for seed in (0, 77):
            want = ref.sample_probabilities(p, 300, seed)
            got = port.sample_raw(p, port.canonicals(seed, 300))
            assert np.array_equal(got, want), (size, seed)
