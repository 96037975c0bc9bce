"""Seeded synthetic workloads: random brickwork circuits, hardware-efficient
ansatz circuits, random Pauli Hamiltonians and the XXZ chain.

Draws come from numpy's PCG64 generator with an explicit seed, except the
random U matrices of `random_layers`, which come from kettle's own
generate_random_unitary2x2 construction on a std::mt19937 stream; the engine,
the oracle and the reference arm see identical gate records.
"""
from __future__ import annotations

import math

import numpy as np

from .capi import GATE_DTYPE, OP, PAULI_DTYPE

TWO_PI = 2.0 * math.pi


def gate(name: str, target: int, control: int = 0, angle: float = 0.0, u=None, param: int = -1):
    rec = np.zeros(1, dtype=GATE_DTYPE)
    rec["op"] = OP[name]
    rec["target"] = target
    rec["control"] = control
    rec["angle"] = angle
    rec["param"] = param
    if u is not None:
        m = np.asarray(u, dtype=np.complex128).reshape(2, 2)
        rec["u"][0] = [m[0, 0].real, m[0, 0].imag, m[0, 1].real, m[0, 1].imag,
                       m[1, 0].real, m[1, 0].imag, m[1, 1].real, m[1, 1].imag]
    return rec


def gates_from_list(items) -> np.ndarray:
    """items: iterables of (name, target[, control[, angle[, u]]]) -> record array."""
    out = np.zeros(len(items), dtype=GATE_DTYPE)
    for i, it in enumerate(items):
        name = it[0]
        out[i] = gate(name, *it[1:])[0]
    return out


def haar_unitary2(rng: np.random.Generator) -> np.ndarray:
    """Haar-random U(2): global phase e^{ia}, |u00| = cos(psi) with psi = asin(sqrt(U[0,1]))."""
    a, phi, chi = TWO_PI * rng.random(3)
    psi = math.asin(math.sqrt(rng.random()))
    g = complex(math.cos(a), math.sin(a))
    ep = complex(math.cos(phi), math.sin(phi))
    ec = complex(math.cos(chi), math.sin(chi))
    c, s = math.cos(psi), math.sin(psi)
    return np.array([[g * c * ep, g * s * ec], [-g * s / ec, g * c / ep]], dtype=np.complex128)


def random_unitaries(seed: int, count: int) -> list[np.ndarray]:
    """`count` Haar-random 2x2 unitaries drawn one after another from one
    std::mt19937(seed) stream, as kettle's
    generate_random_unitary2x2(std::mt19937&) draws them
    (gates/random_u_gates.cpp:13-36): four uniform_real_distribution{0, 1}
    values per matrix (alpha, phi, chi, then psi = asin(sqrt(u))), each one
    std::generate_canonical<double, 53> of the engine (two 32-bit outputs),
    and the same products and quotients:
        U = [[g cos(psi) e^{i phi},  g sin(psi) e^{i chi}],
             [-g sin(psi) / e^{i chi}, g cos(psi) / e^{i phi}]],  g = e^{i alpha}.
    The canonicals come from the library's host code (kt_canonicals_mt19937)."""
    from .capi import canonicals_mt19937

    u = canonicals_mt19937(seed, 4 * count)
    out = []
    for k in range(count):
        alpha = 2.0 * math.pi * float(u[4 * k])
        phi = 2.0 * math.pi * float(u[4 * k + 1])
        chi = 2.0 * math.pi * float(u[4 * k + 2])
        psi = math.asin(math.sqrt(float(u[4 * k + 3])))
        cp, sp = math.cos(psi), math.sin(psi)
        g = complex(math.cos(alpha), math.sin(alpha))
        ep = complex(math.cos(phi), math.sin(phi))
        ec = complex(math.cos(chi), math.sin(chi))
        out.append(np.array([[g * cp * ep, g * sp * ec], [-g * sp / ec, g * cp / ep]], dtype=np.complex128))
    return out


def random_layers(n: int, layers: int, seed: int, mixed: bool = False) -> np.ndarray:
    """The random-circuit family of the benchmark configurations.

    Each layer: one gate per qubit drawn uniformly from {H, RX, RY, RZ}
    (plus U when `mixed`), angles uniform in [0, 2pi); then CX on
    (0,1),(2,3),... on even layers and (1,2),(3,4),... on odd layers; when
    `mixed`, then n//2 controlled rotations drawn from {CRX, CRY, CRZ, CP} on
    random distinct (control, target) pairs with angles uniform in [0, 2pi).
    Gate choices, qubits and angles come from numpy's PCG64(seed); the U
    matrices, in circuit order, from kettle's own generator on one
    std::mt19937(seed) stream (`random_unitaries`), so a kettle program
    seeding std::mt19937 with the same value draws the same matrices.
    """
    rng = np.random.default_rng(seed)
    # at most one U per one-qubit slot: the stream's first layers * n matrices
    u_stream = iter(random_unitaries(seed, layers * n)) if mixed else iter(())
    one_q = ["H", "RX", "RY", "RZ"] + (["U"] if mixed else [])
    ctl = ["CRX", "CRY", "CRZ", "CP"]
    recs = []
    for layer in range(layers):
        for q in range(n):
            name = one_q[int(rng.integers(len(one_q)))]
            if name == "H":
                recs.append(gate("H", q))
            elif name == "U":
                recs.append(gate("U", q, u=next(u_stream)))
            else:
                recs.append(gate(name, q, angle=float(TWO_PI * rng.random())))
        for q in range(layer % 2, n - 1, 2):
            recs.append(gate("CX", q + 1, control=q))
        if mixed:
            for _ in range(n // 2):
                c, t = rng.choice(n, size=2, replace=False)
                name = ctl[int(rng.integers(len(ctl)))]
                recs.append(gate(name, int(t), control=int(c), angle=float(TWO_PI * rng.random())))
    return np.concatenate(recs) if recs else np.zeros(0, dtype=GATE_DTYPE)


def gates_per_layer(n: int, mixed: bool) -> float:
    """Average gate count of one layer of `random_layers` (even and odd layers alternate)."""
    cx = ((n // 2) + ((n - 1) // 2)) / 2.0
    return n + cx + (n // 2 if mixed else 0)


def hea(n: int, layers: int, seed: int):
    """Hardware-efficient ansatz: per layer RY(theta) on every qubit, RZ(theta)
    on every qubit, then CZ on the ring (q, q+1 mod n).  Every rotation has
    its own parameter slot; parameters uniform in [-pi, pi).

    Returns (gates, params)."""
    rng = np.random.default_rng(seed)
    recs = []
    slot = 0
    for _ in range(layers):
        for name in ("RY", "RZ"):
            for q in range(n):
                recs.append(gate(name, q, param=slot))
                slot += 1
        for q in range(n):
            recs.append(gate("CZ", (q + 1) % n, control=q))
    params = rng.uniform(-math.pi, math.pi, size=slot)
    return np.concatenate(recs), params


def pauli(n: int, terms: dict[int, str], phase: int = 0) -> np.ndarray:
    rec = np.zeros(1, dtype=PAULI_DTYPE)
    x = z = 0
    for q, p in terms.items():
        if p in ("X", "Y"):
            x |= 1 << q
        if p in ("Z", "Y"):
            z |= 1 << q
    rec["x"] = x
    rec["z"] = z
    rec["phase"] = phase
    return rec


def random_paulis(n: int, count: int, seed: int):
    """`count` random strings (each site uniform over I/X/Y/Z) with N(0,1) real coefficients.

    Returns (strings, coeffs complex128)."""
    rng = np.random.default_rng(seed)
    out = np.zeros(count, dtype=PAULI_DTYPE)
    for k in range(count):
        sites = rng.integers(4, size=n)
        x = z = 0
        for q, s in enumerate(sites):
            if s in (1, 2):
                x |= 1 << q
            if s in (2, 3):
                z |= 1 << q
        out[k]["x"] = x
        out[k]["z"] = z
    coeffs = rng.standard_normal(count).astype(np.complex128)
    return out, coeffs


def xxz_chain(n: int, seed: int, delta: float = 0.5, j: float = 1.0):
    """H = J sum_{i<n-1} (X_i X_{i+1} + Y_i Y_{i+1} + delta Z_i Z_{i+1}) + sum_i h_i Z_i,
    h_i uniform in [-1, 1] (open boundary).  Returns (strings, coeffs)."""
    rng = np.random.default_rng(seed)
    h = rng.uniform(-1.0, 1.0, size=n)
    strs, cs = [], []
    for i in range(n - 1):
        for p, c in (("X", j), ("Y", j), ("Z", j * delta)):
            strs.append(pauli(n, {i: p, i + 1: p}))
            cs.append(c)
    for i in range(n):
        strs.append(pauli(n, {i: "Z"}))
        cs.append(h[i])
    return np.concatenate(strs), np.asarray(cs, dtype=np.complex128)


def hea_batch(count: int, seed: int, qubits=(10, 22), layers=(2, 10), n_strings: int = 50):
    """`count` hardware-efficient-ansatz instances with qubit counts uniform
    over `qubits` and depths uniform over `layers` (inclusive), each with its
    own parameters (uniform in [-pi, pi)) and its own Hamiltonian of
    `n_strings` random Pauli strings with N(0,1) coefficients.

    Returns (circuits, params): circuits is a list of
    (n_qubits, gates, n_params, strings, coeffs) in the form
    kettle_b200.capi.batch_items takes; params is the concatenated vector."""
    rng = np.random.default_rng(seed)
    circuits, params = [], []
    for b in range(count):
        n = int(rng.integers(qubits[0], qubits[1] + 1))
        d = int(rng.integers(layers[0], layers[1] + 1))
        sub = int(rng.integers(1 << 31))
        gates, p = hea(n, d, seed=sub)
        strings, coeffs = random_paulis(n, n_strings, seed=sub + 1)
        circuits.append((n, gates, p.size, strings, coeffs))
        params.append(p)
    return circuits, np.concatenate(params)
