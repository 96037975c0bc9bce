"""Generate the golden fixtures in tests/golden/ (run once, in a container where
the reference has been compiled into oracle/_ref by `make -C oracle ref`):

    python tests/golden/make_golden.py

    python tests/golden/make_golden.py dm_ops     # golden_dm_ops.npz only
    python tests/golden/make_golden.py size       # golden_size.npz only (~1 min)

Writes
  * ref_kats.json   known-answer cases restated from the reference's own tests
                    (file:line cited per case), expected values as the tests
                    state them;
  * golden_ref.npz  outputs of the reference library itself (oracle/_ref) on
                    seeded small workloads: pair sequences, final amplitudes,
                    expectation values, sampled indices, M-gate outcomes and
                    density matrices;
  * golden_dm_ops.npz partial traces, tensor products and Tr(rho^2) of the
                    reference library on seeded random density matrices;
  * golden_size.npz the 20-qubit, 100-layer benchmark configuration in full
                    (probe amplitudes, state sums, all 200 <P_k>, 4096 shots)
                    and a stream of generate_random_unitary2x2 matrices.
The fixtures are committed; tests read them without needing the reference.
"""
from __future__ import annotations

import json
import math
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from kettle_b200 import workloads as W  # noqa: E402
from oracle.oracle import ref  # noqa: E402

HERE = pathlib.Path(__file__).resolve().parent
S = 1.0 / math.sqrt(2.0)


def basis(n, bits_le: str):
    """Little-endian bitstring (character i = qubit i) -> amplitude vector."""
    v = np.zeros(1 << n, dtype=np.complex128)
    v[sum(1 << i for i, ch in enumerate(bits_le) if ch == "1")] = 1.0
    return v


def kats():
    cases = []

    def sv(name, cite, n, gates, expected, init=None):
        cases.append({"kind": "sv", "name": name, "cite": cite, "n": n, "gates": gates,
                      "init": None if init is None else [[c.real, c.imag] for c in init],
                      "expected": [[complex(c).real, complex(c).imag] for c in expected]})

    t = "test/source/simulation/simulate_test.cpp"
    sv("X(0) on 1 qubit", f"{t}:190-207", 1, [["X", 0]], [0, 1])
    sv("X(1) on 2 qubits", f"{t}:209-226", 2, [["X", 1]], [0, 0, 1, 0])
    sv("X(0)X(1) on 2 qubits", f"{t}:228-246", 2, [["X", 0], ["X", 1]], [0, 0, 0, 1])
    sv("H(0) on 1 qubit", f"{t}:251-268", 1, [["H", 0]], [S, S])
    sv("H(0) on 2 qubits", f"{t}:270-287", 2, [["H", 0]], [S, S, 0, 0])
    sv("H(1) on 2 qubits", f"{t}:289-306", 2, [["H", 1]], [S, 0, S, 0])
    sv("H(0)H(1) on 2 qubits", f"{t}:308-327", 2, [["H", 0], ["H", 1]], [0.5, 0.5, 0.5, 0.5])
    # gate definitions the tests rely on (gates/common_u_gates.cpp:120-170 matrices)
    for th in (0.0, math.pi / 3, math.pi, 2.5):
        c, s = math.cos(th / 2), math.sin(th / 2)
        sv(f"RX({th:.4f}) |0>", f"{t}:330-420 (RX family)", 1, [["RX", 0, 0, th]], [c, -1j * s])
        sv(f"RY({th:.4f}) |0>", f"{t}:420-520 (RY family)", 1, [["RY", 0, 0, th]], [c, s])
        sv(f"RZ({th:.4f}) |+>", f"{t}:520-620 (RZ family)", 1, [["RZ", 0, 0, th]],
           [S * complex(c, -s), S * complex(c, s)], init=[S, S])
        sv(f"P({th:.4f}) |1>", f"{t} (P family)", 1, [["P", 0, 0, th]], [0, complex(math.cos(th), math.sin(th))],
           init=[0, 1])
    sv("CX(0->1) |10>", f"{t}:620-700 (CX family)", 2, [["CX", 1, 0]], basis(2, "11"), init=basis(2, "10"))
    sv("CX(0->1) |00>", f"{t}:620-700 (CX family)", 2, [["CX", 1, 0]], basis(2, "00"), init=basis(2, "00"))
    sv("CZ(0,1) |11>", f"{t}:700-760 (CZ family)", 2, [["CZ", 1, 0]], -basis(2, "11"), init=basis(2, "11"))
    sv("H(0) CX(0->1): Bell", "README.md:37-60", 2, [["H", 0], ["CX", 1, 0]], [S, 0, 0, S])
    # Pauli strings applied to basis states (test/source/simulation/simulate_pauli_test.cpp:10-88)
    p = "test/source/simulation/simulate_pauli_test.cpp"
    pa = []
    pa.append({"name": "empty", "cite": f"{p}:12-22", "n": 3, "terms": {}, "init": "000", "out": "000", "factor": [1, 0]})
    pa.append({"name": "X0", "cite": f"{p}:24-34", "n": 3, "terms": {"0": "X"}, "init": "000", "out": "100", "factor": [1, 0]})
    pa.append({"name": "X0 X2", "cite": f"{p}:36-47", "n": 3, "terms": {"0": "X", "2": "X"}, "init": "000", "out": "101",
               "factor": [1, 0]})
    pa.append({"name": "Y1", "cite": f"{p}:49-60", "n": 3, "terms": {"1": "Y"}, "init": "000", "out": "010", "factor": [0, 1]})
    pa.append({"name": "Z1 on 010", "cite": f"{p}:62-73", "n": 3, "terms": {"1": "Z"}, "init": "010", "out": "010",
               "factor": [-1, 0]})
    pa.append({"name": "X0 Y1 Z2 on 011", "cite": f"{p}:75-87", "n": 3, "terms": {"0": "X", "1": "Y", "2": "Z"},
               "init": "011", "out": "101", "factor": [0, 1]})
    # expectation values (test/source/operator/pauli/pauli_operator_test.cpp)
    q = "test/source/operator/pauli/pauli_operator_test.cpp"
    one = {"x+": [S, S], "x-": [S, -S], "y+": [S, 1j * S], "y-": [S, -1j * S], "z+": [1, 0], "z-": [0, 1]}
    table1 = [("X", "x+", 1), ("X", "x-", -1), ("X", "y+", 0), ("X", "y-", 0), ("X", "z+", 0), ("X", "z-", 0),
              ("Y", "x+", 0), ("Y", "x-", 0), ("Y", "y+", 1), ("Y", "y-", -1), ("Y", "z+", 0), ("Y", "z-", 0),
              ("Z", "x+", 0), ("Z", "x-", 0), ("Z", "y+", 0), ("Z", "y-", 0), ("Z", "z+", 1), ("Z", "z-", -1)]
    ex = []
    for term, st, val in table1:
        ex.append({"cite": f"{q}:18-61", "n": 1, "state": [[complex(c).real, complex(c).imag] for c in one[st]],
                   "ops": [[[1, 0], {"0": term}]], "expected": [val, 0]})

    def kron_le(a, b):
        # tensor_product(left, right): left qubit 0 (state.cpp:141-155): index = i_left + n_left * i_right
        return np.kron(np.asarray(b, dtype=complex), np.asarray(a, dtype=complex))

    table2 = [("Z", "Z", "z+", "z+", 1), ("Z", "Z", "z+", "z-", -1), ("Z", "Z", "z-", "z+", -1), ("Z", "Z", "z-", "z-", 1),
              ("X", "X", "z+", "z+", 0), ("X", "X", "z+", "z-", 0), ("X", "X", "z-", "z+", 0), ("X", "X", "z-", "z-", 0),
              ("X", "Z", "x+", "z+", 1), ("X", "Z", "x+", "z-", -1), ("X", "X", "x+", "z+", 0), ("X", "X", "x+", "x-", -1)]
    for t0, t1, s0, s1, val in table2:
        st = kron_le(one[s0], one[s1])
        ex.append({"cite": f"{q}:64-101", "n": 2, "state": [[c.real, c.imag] for c in st],
                   "ops": [[[1, 0], {"0": t0, "1": t1}]], "expected": [val, 0]})
    ex.append({"cite": f"{q}:105-117", "n": 1, "state": [[1, 0], [0, 0]],
               "ops": [[[1, 0], {"0": "Z"}], [[1, 0], {"0": "X"}]], "expected": [1, 0]})
    ex.append({"cite": f"{q}:119-131", "n": 1, "state": [[S, 0], [S, 0]],
               "ops": [[[1, 0], {"0": "Z"}], [[-2, 0], {"0": "X"}]], "expected": [-2, 0]})
    bell = [S, 0, 0, S]
    ex.append({"cite": f"{q}:133-154", "n": 2, "state": [[c, 0] for c in bell],
               "ops": [[[1, 0], {"0": "Z", "1": "Z"}], [[1, 0], {"0": "X", "1": "X"}]], "expected": [2, 0]})
    ghz = np.zeros(8)
    ghz[0] = ghz[7] = S
    ex.append({"cite": f"{q}:156-178", "n": 3, "state": [[c, 0] for c in ghz],
               "ops": [[[1, 0], {"0": "Z", "1": "Z", "2": "Z"}], [[1, 0], {"0": "X", "1": "X", "2": "X"}]],
               "expected": [1, 0]})
    pp = [0.5, 0.5, 0.5, 0.5]
    ex.append({"cite": f"{q}:180-200", "n": 2, "state": [[c, 0] for c in pp],
               "ops": [[[1, 0], {"0": "X"}], [[0, -1], {"1": "X"}]], "expected": [1, -1]})
    cdf = {"cite": "test/source/calculations/probabilities_test.cpp:21-30", "probs": [0.25] * 4,
           "cdf": [0.25, 0.5, 0.75, 1.0]}
    return {"sv": cases, "pauli_apply": pa, "expect": ex, "cdf": cdf}


def golden_ref():
    R = ref()
    out = {}
    # pair sequences (reference order) for small n, every target / (control, target)
    for n in range(1, 7):
        for t in range(n):
            out[f"pairs_s_{n}_{t}"] = R.pairs_single(n, t)
            if n >= 2:
                for c in range(n):
                    if c != t:
                        out[f"pairs_d_{n}_{c}_{t}"] = R.pairs_double(n, c, t, quad=False)
                        out[f"pairs_q_{n}_{c}_{t}"] = R.pairs_double(n, c, t, quad=True)
    # the set_state() windows of gate_pair_generator_test.cpp:400-473
    for a, b in ((10, 15), (7, 10), (3, 7), (0, 5), (9, 13)):
        out[f"pairs_ss_5_3_{a}_{b}"] = R.pairs_single(5, 3, k0=a, count=b - a)
        out[f"pairs_ds_6_2_3_{a}_{b}"] = R.pairs_double(6, 2, 3, k0=a, count=b - a)
    # random circuits: final amplitudes from |0...0>
    for n, layers, mixed, seed in ((6, 8, False, 11), (6, 6, True, 12), (10, 10, False, 13), (10, 6, True, 14)):
        g = W.random_layers(n, layers, seed=seed, mixed=mixed)
        a, _ = R.simulate_sv(n, basis(n, "0" * n), g)
        out[f"circ_{n}_{layers}_{int(mixed)}_{seed}_gates"] = g
        out[f"circ_{n}_{layers}_{int(mixed)}_{seed}_amps"] = a
        strs, cf = W.random_paulis(n, 25, seed=seed + 100)
        terms, total = R.expect(n, a, strs, cf)
        out[f"circ_{n}_{layers}_{int(mixed)}_{seed}_strings"] = strs
        out[f"circ_{n}_{layers}_{int(mixed)}_{seed}_coeffs"] = cf
        out[f"circ_{n}_{layers}_{int(mixed)}_{seed}_terms"] = terms
        out[f"circ_{n}_{layers}_{int(mixed)}_{seed}_total"] = np.array([total])
        for shots_seed in (1, 42):
            out[f"circ_{n}_{layers}_{int(mixed)}_{seed}_samples_{shots_seed}"] = R.sample_memory(n, a, 512, shots_seed)
    # parameterised circuit with shared parameters
    g, params = W.hea(5, 3, seed=21)
    g["param"][10] = 0  # a second gate bound to parameter 0
    a, _ = R.simulate_sv(5, basis(5, "00000"), g, params=params)
    out["hea_5_3_gates"] = g
    out["hea_5_3_params"] = params
    out["hea_5_3_amps"] = a
    # M gates: outcome and collapsed state per seed
    n = 5
    g = W.random_layers(n, 3, seed=31, mixed=True)
    a0, _ = R.simulate_sv(n, basis(n, "0" * n), g)
    out["meas_pre_amps"] = a0
    ms, mo, ma = [], [], []
    for seed in range(12):
        qb = seed % n
        gm = W.gate("M", qb, control=qb)
        a1, cb = R.simulate_sv(n, a0, gm, seed=seed)
        ms.append([seed, qb])
        mo.append(cb[qb])
        ma.append(a1)
    out["meas_seed_qubit"] = np.array(ms)
    out["meas_outcome"] = np.array(mo)
    out["meas_amps"] = np.array(ma)
    # density matrix
    for n, layers, seed in ((3, 3, 41), (4, 2, 42)):
        g = W.random_layers(n, layers, seed=seed, mixed=True)
        rho0 = np.zeros((1 << n, 1 << n), dtype=np.complex128)
        rho0[0, 0] = 1.0
        out[f"dm_{n}_{layers}_{seed}_gates"] = g
        out[f"dm_{n}_{layers}_{seed}_rho"] = R.simulate_dm(n, rho0, g)
    # probabilities with readout noise
    n = 6
    a = out["circ_6_8_0_11_amps"]
    noise = np.linspace(0.0, 0.25, n)
    out["noise_vec"] = noise
    out["noise_probs"] = R.probabilities(n, a, noise)
    return out


CONFIG1_SEED = 2024          # the seed the benchmark draws its workloads with
CONFIG1_PROBES = 4096        # amplitudes kept per state (the full 20-qubit state is 16 MiB)


def golden_size():
    """Full-size fixtures of the reference library:
      * config 1 in full: the 20-qubit complex128 state after all 100 layers
        (2950 gates) of the benchmark circuit, then <P_k> of all 200 strings,
        the weighted total and 4096 sampled indices (std::mt19937(2024)
        through perform_measurements_as_memory); the state is kept as
        amplitudes at CONFIG1_PROBES seeded indices plus two sums over every
        amplitude (sum |a_i|^2 i and sum a_i e^{-2 pi i i / 2^20 * 7}), so a
        tile placed at the wrong address changes them;
      * generate_random_unitary2x2 on one std::mt19937 stream (the source of
        the benchmark circuits' U gates)."""
    R = ref()
    out = {}
    n = 20
    gates = W.random_layers(n, 100, seed=CONFIG1_SEED, mixed=False)
    strings, coeffs = W.random_paulis(n, 200, seed=CONFIG1_SEED)
    amps, _ = R.simulate_sv(n, basis(n, "0" * n), gates)
    terms, total = R.expect(n, amps, strings, coeffs)
    out["c1_gates"] = gates
    out["c1_strings"] = strings
    out["c1_coeffs"] = coeffs
    out["c1_terms"] = terms
    out["c1_total"] = np.array([total])
    out["c1_samples"] = R.sample_memory(n, amps, 4096, CONFIG1_SEED)
    idx = np.random.default_rng(7).choice(1 << n, size=CONFIG1_PROBES, replace=False).astype(np.int64)
    out["c1_probe_index"] = idx
    out["c1_probe_amps"] = amps[idx]
    out["c1_sums"] = np.array(state_sums(amps))
    for seed in (0, 2024):
        out[f"ru_{seed}"] = np.array(R.random_unitaries(seed, 64))
    return out


def state_sums(amps):
    """Two sums over every amplitude: sum |a_i|^2 i and sum a_i w^(7 i) with
    w = e^{-2 pi i / N} (a single Fourier coefficient)."""
    N = amps.size
    i = np.arange(N, dtype=np.float64)
    s1 = float(np.sum(np.abs(amps) ** 2 * i))
    s2 = complex(np.sum(amps * np.exp(-2j * np.pi * 7.0 * i / N)))
    return [s1, s2.real, s2.imag]


def random_rho(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((1 << n, 1 << n)) + 1j * rng.standard_normal((1 << n, 1 << n))
    rho = a @ a.conj().T
    return rho / np.trace(rho)


# traced-qubit lists per size: single qubits, several in either order, a
# repeated index (read as the reference reads it) and every qubit
DM_TRACE_CASES = {
    3: [[0], [1], [2], [0, 2], [2, 0], [1, 1], [0, 1, 2]],
    4: [[3], [0, 3], [3, 1, 0], [2, 2], [0, 1, 2, 3]],
    5: [[2], [4, 0], [1, 3], [0, 2, 4], [3, 3, 1]],
}


def golden_dm_ops():
    """Partial traces, tensor products and Tr(rho^2) of the reference library
    (state/density_matrix.cpp:187-278) on seeded random density matrices."""
    R = ref()
    out = {}
    for n, cases in DM_TRACE_CASES.items():
        rho = random_rho(n, 100 + n)
        out[f"dmop_{n}_rho"] = rho
        out[f"dmop_{n}_tsq"] = np.array([R.dm_trace_of_square(n, rho)])
        for j, qs in enumerate(cases):
            out[f"dmop_{n}_pt_{j}_q"] = np.array(qs, dtype=np.int64)
            out[f"dmop_{n}_pt_{j}_out"] = R.dm_partial_trace(n, rho, qs)
    left, right = random_rho(2, 7), random_rho(3, 8)
    out["dmop_tp_left"] = left
    out["dmop_tp_right"] = right
    out["dmop_tp_out"] = R.dm_tensor_product(2, left, 3, right)
    return out


def main():
    which = sys.argv[1:] or ["all"]
    if "all" in which:
        (HERE / "ref_kats.json").write_text(json.dumps(kats(), indent=1))
        np.savez_compressed(HERE / "golden_ref.npz", **golden_ref())
        print("wrote", HERE / "ref_kats.json", HERE / "golden_ref.npz")
    if "all" in which or "dm_ops" in which:
        np.savez_compressed(HERE / "golden_dm_ops.npz", **golden_dm_ops())
        print("wrote", HERE / "golden_dm_ops.npz")
    if "all" in which or "size" in which:
        np.savez_compressed(HERE / "golden_size.npz", **golden_size())
        print("wrote", HERE / "golden_size.npz")


if __name__ == "__main__":
    main()
