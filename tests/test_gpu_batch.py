"""Batch engine (kt_batch) against the single-circuit adjoint path, item by
item: same energies and gradients (1e-10, complex128) for items that run in
shared memory, items that run from HBM in the persistent work-queue kernel
and items that run run-time compiled block kernels shared by their plan
structure class, across graph replays with new parameters, with shared
parameter slots, without gradients, and in complex64 (1e-3 of complex128)."""
import numpy as np
import pytest

from conftest import basis
from kettle_b200 import capi
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _mixed(n, seed, layers=3):
    """Rotations (plain and controlled), CX, H, Haar U and literal-angle gates."""
    rng = np.random.default_rng(seed)
    recs, slot = [], 0
    names = ["RX", "RY", "RZ", "P", "CRX", "CRY", "CRZ", "CP"]
    for layer in range(layers):
        for q in range(n):
            recs.append(W.gate(names[int(rng.integers(4))], q, param=slot))
            slot += 1
        for _ in range(n // 2):
            c, t = rng.choice(n, 2, replace=False)
            recs.append(W.gate(names[4 + int(rng.integers(4))], int(t), control=int(c), param=slot))
            slot += 1
        for q in range(layer % 2, n - 1, 2):
            recs.append(W.gate("CX", q + 1, control=q))
        recs.append(W.gate("U", int(rng.integers(n)), u=W.haar_unitary2(rng)))
        recs.append(W.gate("H", int(rng.integers(n))))
        recs.append(W.gate("RX", int(rng.integers(n)), angle=0.3))
    return np.concatenate(recs), rng.uniform(-np.pi, np.pi, slot)


def _items(seed=5):
    """Small (shared-memory) and large (HBM) items of both circuit families."""
    circuits, params = [], []
    spec = [(5, "hea"), (9, "mixed"), (12, "hea"), (13, "hea"), (14, "mixed"), (15, "hea"), (13, "empty"), (3, "mixed")]
    for k, (n, kind) in enumerate(spec):
        if kind == "hea":
            g, p = W.hea(n, 2 + k % 3, seed=seed + k)
        elif kind == "mixed":
            g, p = _mixed(n, seed + k)
        else:
            g, p = np.zeros(0, dtype=capi.GATE_DTYPE), np.zeros(0)
        s, c = W.random_paulis(n, 12 + k, seed=seed + 100 + k)
        circuits.append((n, g, p.size, s, c))
        params.append(p)
    return circuits, np.concatenate(params)


def _one_by_one(circuits, params, dtype=capi.KT_C128):
    es, gs, off = [], [], 0
    for n, g, np_, s, c in circuits:
        p = params[off:off + np_]
        off += np_
        sv = capi.Statevector(n, dtype)
        adj = capi.Adjoint(sv)
        es.append(adj.forward(g, p, s, c))
        gs.append(adj.backward() if np_ else np.zeros(0))
        adj.close()
        sv.close()
    return np.array(es), np.concatenate(gs)


def test_batch_matches_single_circuit_path(engine):
    circuits, params = _items()
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    b = capi.Batch(items, gates, strings, coeffs, n_params)
    st = b.stats()
    assert st["small_items"] == 4 and st["large_items"] == 4
    e, g = b.evaluate(params)
    e1, g1 = _one_by_one(circuits, params)
    assert np.abs(e - e1).max() < 1e-10
    assert np.abs(g - g1).max() < 1e-10
    # the empty 13-qubit item: E = <0|H|0> = sum of the coefficients of the Z-only strings
    n, _, _, s, c = circuits[6]
    z_only = (s["x"] == 0)
    assert abs(e[6] - c[z_only].real.sum()) < 1e-12
    # replay with new parameters
    p2 = np.random.default_rng(1).uniform(-np.pi, np.pi, params.size)
    e2, g2 = b.evaluate(p2)
    e3, g3 = _one_by_one(circuits, p2)
    assert np.abs(e2 - e3).max() < 1e-10 and np.abs(g2 - g3).max() < 1e-10
    b.close()


def test_batch_energy_against_oracle(engine, port):
    circuits, params = _items()
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    b = capi.Batch(items, gates, strings, coeffs, n_params, with_grad=False)
    e, g = b.evaluate(params)
    assert g is None
    off = 0
    for k, (n, gk, np_, s, c) in enumerate(circuits):
        if n <= 13:
            psi = port.apply(n, basis(n), gk, params[off:off + np_])
            ref = port.expect(n, psi, s, c)[1].real
            assert abs(e[k] - ref) < 1e-11, k
        off += np_
    b.close()


def test_batch_shared_parameters_sum(engine):
    n = 13
    g, p = W.hea(n, 3, seed=9)
    s1, c1 = W.random_paulis(n, 10, seed=1)
    s2, c2 = W.random_paulis(n, 10, seed=2)
    items = np.zeros(3, dtype=capi.BATCH_ITEM_DTYPE)
    # items 0 and 1 share one parameter range; item 2 is a small copy of item 0 on its own range
    gs, ps = W.hea(6, 2, seed=3)
    s3, c3 = W.random_paulis(6, 8, seed=3)
    gates = np.concatenate([g, gs])
    strings = np.concatenate([s1, s2, s3])
    coeffs = np.concatenate([c1, c2, c3])
    items[0] = (n, 0, 0, g.size, 0, p.size, 0, s1.size)
    items[1] = (n, 0, 0, g.size, 0, p.size, s1.size, s2.size)
    items[2] = (6, 0, g.size, gs.size, p.size, ps.size, s1.size + s2.size, s3.size)
    b = capi.Batch(items, gates, strings, coeffs, p.size + ps.size)
    e, grad = b.evaluate(np.concatenate([p, ps]))
    ea, ga = _one_by_one([(n, g, p.size, s1, c1)], p)
    eb, gb = _one_by_one([(n, g, p.size, s2, c2)], p)
    ec, gc = _one_by_one([(6, gs, ps.size, s3, c3)], ps)
    assert abs(e[0] - ea[0]) < 1e-10 and abs(e[1] - eb[0]) < 1e-10 and abs(e[2] - ec[0]) < 1e-10
    assert np.abs(grad[:p.size] - (ga + gb)).max() < 1e-10
    assert np.abs(grad[p.size:] - gc).max() < 1e-10
    b.close()


def test_batch_complex64(engine):
    circuits, params = _items(seed=11)
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    b128 = capi.Batch(items, gates, strings, coeffs, n_params)
    b64 = capi.Batch(items, gates, strings, coeffs, n_params, dtype=capi.KT_C64)
    st = b64.stats()
    assert st["small_items"] == 6 and st["large_items"] == 2   # complex64 keeps 13 qubits in shared memory
    e0, g0 = b128.evaluate(params)
    e1, g1 = b64.evaluate(params)
    assert np.abs(e0 - e1).max() < 1e-3
    assert np.abs(g0 - g1).max() < 1e-3
    b128.close()
    b64.close()


def test_batch_run_one_shot(engine):
    circuits, params = _items(seed=21)
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    b = capi.Batch(items, gates, strings, coeffs, n_params)
    e0, g0 = b.evaluate(params)
    b.close()
    import ctypes as C
    e = np.empty(items.size)
    g = np.empty(n_params)
    it = np.ascontiguousarray(items)
    gg = np.ascontiguousarray(gates)
    ss = np.ascontiguousarray(strings)
    cc = np.ascontiguousarray(coeffs)
    capi.check(capi.lib().kt_batch_run(capi.ptr(it), it.size, capi.ptr(gg), gg.size, capi.ptr(params), params.size,
                                       capi.ptr(ss), capi.ptr(cc), ss.size, capi.KT_C128, capi.ptr(e), capi.ptr(g),
                                       None))
    assert np.array_equal(e, e0) and np.array_equal(g, g0)


def test_batch_many_items_work_queue(engine):
    """A few hundred HEA items of 10..16 qubits: many HBM items in flight at once."""
    circuits, params = W.hea_batch(300, seed=4, qubits=(10, 16), layers=(2, 5), n_strings=10)
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    b = capi.Batch(items, gates, strings, coeffs, n_params)
    e, g = b.evaluate(params)
    sel = list(range(0, len(circuits), 23))
    off = np.cumsum([0] + [c[2] for c in circuits])
    for k in sel:
        e1, g1 = _one_by_one([circuits[k]], params[off[k]:off[k + 1]])
        assert abs(e[k] - e1[0]) < 1e-10
        assert np.abs(g[off[k]:off[k + 1]] - g1).max() < 1e-10
    b.close()


def test_batch_wait_limit_returns_timeout_and_the_context_stays_usable(engine):
    """The persistent kernel's bounded wait: with batch_spin_limit at a few
    polls, CTAs that find no ready job (most of them, while the first forward
    blocks run) give up at once; the evaluation stops with KT_ERR_TIMEOUT, the
    kernel returns, and a batch created afterwards with the default limit
    evaluates normally on the same context."""
    circuits = []
    params = []
    for k, n in enumerate((16, 17, 16)):
        g, p = W.hea(n, 6, seed=70 + k)
        s, c = W.random_paulis(n, 20, seed=80 + k)
        circuits.append((n, g, p.size, s, c))
        params.append(p)
    params = np.concatenate(params)
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    old = capi.tuning_get("batch_spin_limit")
    old_jit = capi.tuning_get("batch_jit_min_qubits")
    capi.tuning_set("batch_spin_limit", 2)
    capi.tuning_set("batch_jit_min_qubits", 0)  # these items run in the persistent kernel
    try:
        b = capi.Batch(items, gates, strings, coeffs, n_params)
    finally:
        capi.tuning_set("batch_spin_limit", old)
        capi.tuning_set("batch_jit_min_qubits", old_jit)
    with pytest.raises(capi.KettleError) as e:
        b.evaluate(params)
    assert e.value.code == capi.KT_ERR_TIMEOUT
    b.close()
    b2 = capi.Batch(items, gates, strings, coeffs, n_params)
    energies, grads = b2.evaluate(params)
    b2.close()
    want_e, want_g = _one_by_one(circuits, params)
    assert np.abs(energies - want_e).max() < 1e-10
    assert np.abs(grads - want_g).max() < 1e-10


def _with_knob(name, value, fn):
    old = capi.tuning_get(name)
    capi.tuning_set(name, value)
    try:
        return fn()
    finally:
        capi.tuning_set(name, old)


def _class_items(seed):
    """HBM items in repeated structures: HEA at 14, 15 and 17 qubits (four
    items each, own parameters and Hamiltonians), a mixed-gate circuit at 16
    qubits twice, and single items at 13 and 14 qubits."""
    circuits, params = [], []
    spec = [(14, 3)] * 4 + [(15, 2)] * 4 + [(17, 4)] * 4 + [(13, 2), (14, 5)]
    for k, (n, layers) in enumerate(spec):
        g, p = W.hea(n, layers, seed=seed + k)
        s, c = W.random_paulis(n, 10 + k, seed=seed + 50 + k)
        circuits.append((n, g, p.size, s, c))
        params.append(p)
    g, p0 = _mixed(16, seed + 7)
    for k in range(2):
        s, c = W.random_paulis(16, 15, seed=seed + 90 + k)
        circuits.append((16, g, p0.size, s, c))
        params.append(p0 + 0.1 * k)
    return circuits, np.concatenate(params)


def test_batch_compiled_classes_match_single_path(engine):
    """batch_jit_min_qubits = 14: every HBM item of 14 or more qubits runs the
    batched compiled kernels of its class (the four-item HEA groups, the
    mixed circuit pair, single items as classes of one); energies and
    gradients equal the single-circuit path (1e-10) and the persistent
    kernel's (1e-11), on two evaluations with new parameters."""
    circuits, params = _class_items(300)
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    b = _with_knob("batch_jit_min_qubits", 14, lambda: capi.Batch(items, gates, strings, coeffs, n_params))
    st = b.stats()
    assert st["compiled_items"] == 15 and st["compiled_classes"] == 5, st
    p_ref = _with_knob("batch_jit_min_qubits", 0, lambda: capi.Batch(items, gates, strings, coeffs, n_params))
    assert p_ref.stats()["compiled_items"] == 0
    for shift in (0.0, 0.21):
        p = params + shift
        e, g = b.evaluate(p)
        e0, g0 = p_ref.evaluate(p)
        e1, g1 = _one_by_one(circuits, p)
        assert np.abs(e - e1).max() < 1e-10 and np.abs(g - g1).max() < 1e-10
        assert np.abs(e - e0).max() < 1e-11 and np.abs(g - g0).max() < 1e-11
    b.close()
    p_ref.close()


def test_batch_compiled_without_gradients_and_complex64(engine):
    circuits, params = _class_items(400)
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    mk = lambda **kw: _with_knob("batch_jit_min_qubits", 15, lambda: capi.Batch(items, gates, strings, coeffs,
                                                                                n_params, **kw))
    b = mk(with_grad=False)
    assert b.stats()["compiled_items"] == 10
    e, g = b.evaluate(params)
    assert g is None
    e1, _ = _one_by_one(circuits, params)
    assert np.abs(e - e1).max() < 1e-10
    b.close()
    b64 = mk(dtype=capi.KT_C64)
    assert b64.stats()["compiled_items"] == 10
    e64, g64 = b64.evaluate(params)
    b64.close()
    _, g1 = _one_by_one(circuits, params)
    assert np.abs(e64 - e1).max() < 1e-3 and np.abs(g64 - g1).max() < 1e-3


def test_batch_compiled_kernels_shared_between_batches(engine):
    """A second batch of the same plan structures takes its compiled kernels
    from the process-wide cache: it evaluates the same values, also after the
    first batch is destroyed."""
    circuits, params = _class_items(500)
    items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
    mk = lambda: _with_knob("batch_jit_min_qubits", 14, lambda: capi.Batch(items, gates, strings, coeffs, n_params))
    b1 = mk()
    e1, g1 = b1.evaluate(params)
    b2 = mk()
    b1.close()
    e2, g2 = b2.evaluate(params)
    b2.close()
    assert b2 is not b1
    assert np.array_equal(e1, e2) and np.array_equal(g1, g2)
