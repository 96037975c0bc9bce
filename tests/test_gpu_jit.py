"""Run-time compiled block kernels (fused_jit = 1): the same amplitudes as the
oracle (1e-12) and as the precompiled fused kernels (1e-13) on circuits that
exercise every op kind (general, real, RX-like, anti-diagonal, swap, diagonal
on register / thread / tile-external bits) with controls on register, thread
and tile-external bits and folded permutations; kernels are reused for a new
set of angles; parameterised circuits bind their angles at run time."""
import numpy as np
import pytest

from conftest import basis, random_state
from kettle_b200 import capi
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture()
def jit(engine):
    old = capi.tuning_get("fused_jit")
    capi.tuning_set("fused_jit", 1)
    yield capi
    capi.tuning_set("fused_jit", old)


def _apply(n, init, gates, params=None):
    sv = capi.Statevector(n)
    sv.upload(init)
    sv.apply(gates, params)
    out = sv.download()
    sv.close()
    return out


@pytest.mark.parametrize("n,layers,seed", [(10, 6, 1), (14, 5, 2), (17, 4, 3), (20, 3, 4)])
def test_jit_matches_oracle(jit, port, n, layers, seed):
    g = W.random_layers(n, layers, seed=seed, mixed=True)
    init = random_state(n, seed)
    before = capi.jit_stats()
    got = _apply(n, init, g)
    after = capi.jit_stats()
    assert not after["failed"]
    assert after["launches"] > before["launches"]
    assert np.abs(got - port.apply(n, init, g)).max() < 1e-12


def test_jit_matches_precompiled_and_reuses_kernels(jit):
    n = 24
    g = W.random_layers(n, 4, seed=11, mixed=True)
    a = _apply(n, basis(n), g)
    capi.tuning_set("fused_jit", 0)
    b = _apply(n, basis(n), g)
    capi.tuning_set("fused_jit", 1)
    assert np.abs(a - b).max() < 1e-13
    # new angles, same structure: no new kernels
    g2 = g.copy()
    rng = np.random.default_rng(5)
    has_angle = np.isin(g2["op"], [capi.OP[x] for x in capi.ANGLE_GATES])
    g2["angle"][has_angle] = rng.uniform(0, 2 * np.pi, int(has_angle.sum()))
    k0 = capi.jit_stats()["kernels"]
    c = _apply(n, basis(n), g2)
    assert capi.jit_stats()["kernels"] == k0
    capi.tuning_set("fused_jit", 0)
    d = _apply(n, basis(n), g2)
    capi.tuning_set("fused_jit", 1)
    assert np.abs(c - d).max() < 1e-13


def test_jit_parameterised(jit, port):
    n = 16
    gates, params = W.hea(n, 3, seed=4)
    got = _apply(n, basis(n), gates, params)
    assert np.abs(got - port.apply(n, basis(n), gates, params)).max() < 1e-12
    k0 = capi.jit_stats()["kernels"]
    p2 = params + 0.37
    got2 = _apply(n, basis(n), gates, p2)
    assert capi.jit_stats()["kernels"] == k0
    assert np.abs(got2 - port.apply(n, basis(n), gates, p2)).max() < 1e-12


def test_jit_every_gate_kind(jit, port):
    # every gate on low (register / lane), middle (thread) and high (outside the tile) qubits
    n = 18
    rng = np.random.default_rng(7)
    names = [x for x in capi.GATES if x != "M"]
    parts = []
    for name in names:
        for t, c in ((0, 5), (5, 0), (9, 16), (16, 2), (3, 17)):
            if name in ("U", "CU"):
                parts.append(W.gate(name, t, control=c, u=W.haar_unitary2(rng)))
            elif name in capi.ANGLE_GATES:
                parts.append(W.gate(name, t, control=c, angle=float(rng.uniform(0, 2 * np.pi))))
            else:
                parts.append(W.gate(name, t, control=c))
        parts.append(W.gate("H", int(rng.integers(0, n))))
    g = np.concatenate(parts)
    init = random_state(n, 3)
    assert np.abs(_apply(n, init, g) - port.apply(n, init, g)).max() < 1e-12


def test_auto_mode_compiles_on_the_second_apply(engine, port):
    # fused_jit = 2 with jit_after = 2: a circuit structure new to the process
    # runs on the precompiled kernels; its second apply compiles and runs the
    # block kernels
    old = {k: capi.tuning_get(k) for k in ("fused_jit", "jit_min_qubits", "jit_after")}
    try:
        capi.tuning_set("fused_jit", 2)
        capi.tuning_set("jit_min_qubits", 19)
        capi.tuning_set("jit_after", 2)
        n = 19
        g = W.random_layers(n, 3, seed=99, mixed=True)
        s0 = capi.jit_stats()
        a = _apply(n, basis(n), g)
        s1 = capi.jit_stats()
        assert s1["launches"] == s0["launches"] and s1["kernels"] == s0["kernels"]
        b = _apply(n, basis(n), g)
        s2 = capi.jit_stats()
        assert s2["kernels"] > s1["kernels"] and s2["launches"] > s1["launches"]
        want = port.apply(n, basis(n), g)
        assert np.abs(a - want).max() < 1e-12 and np.abs(b - want).max() < 1e-12
        # below jit_min_qubits nothing is compiled
        small = W.random_layers(12, 3, seed=98, mixed=True)
        _apply(12, basis(12), small)
        _apply(12, basis(12), small)
        assert capi.jit_stats()["kernels"] == s2["kernels"]
    finally:
        for k, v in old.items():
            capi.tuning_set(k, v)


@pytest.mark.parametrize("knobs", [
    {"jit_merge_diag": 0}, {"jit_prefetch": 0}, {"jit_skip_io": 0}, {"jit_skip_io": 1}, {"jit_fence": 2},
    {"jit_scale_ops": 0}, {"jit_remat": 0},
    {"fused_tile_bits": 11, "jit_ctas_per_sm": 3}, {"fused_tile_bits": 13},
])
def test_jit_variants_agree(jit, port, knobs):
    # every generated-kernel variant computes the same state
    old = {k: capi.tuning_get(k) for k in knobs}
    try:
        for k, v in knobs.items():
            capi.tuning_set(k, v)
        n = 18
        g = W.random_layers(n, 4, seed=31, mixed=True)
        init = random_state(n, 31)
        assert np.abs(_apply(n, init, g) - port.apply(n, init, g)).max() < 1e-12
    finally:
        for k, v in old.items():
            capi.tuning_set(k, v)


@pytest.mark.parametrize("renorm", [1, 0])
def test_jit_complex64(jit, port, renorm):
    # complex64 blocks compile too, with the per-block renormalisation by default
    old = capi.tuning_get("c64_renormalize")
    try:
        capi.tuning_set("c64_renormalize", renorm)
        n = 20
        g = W.random_layers(n, 6, seed=41, mixed=True)
        want = port.apply(n, basis(n), g)
        s0 = capi.jit_stats()
        sv = capi.Statevector(n, capi.KT_C64)
        sv.apply(g)
        got = sv.download()
        assert capi.jit_stats()["launches"] > s0["launches"]
        assert np.abs(got - want).max() < 1e-4
        assert abs(sv.norm_sq() - 1.0) < 1e-5
        sv.close()
        capi.tuning_set("fused_jit", 0)
        ref = capi.Statevector(n, capi.KT_C64)
        ref.apply(g)
        assert np.abs(ref.download() - got).max() < 1e-5
        ref.close()
    finally:
        capi.tuning_set("c64_renormalize", old)


def test_jit_density_matrix(jit):
    # a density matrix applies U on its row bits and conj(U) on its column
    # bits through the same fused planner; compiled blocks agree with the
    # precompiled ones
    n = 9
    g = W.random_layers(n, 3, seed=51, mixed=True)
    dm = capi.DensityMatrix(n)
    dm.apply(g)
    a = dm.download()
    capi.tuning_set("fused_jit", 0)
    ref = capi.DensityMatrix(n)
    ref.apply(g)
    b = ref.download()
    capi.tuning_set("fused_jit", 1)
    assert np.abs(a - b).max() < 1e-13
    assert abs(np.trace(a) - 1.0) < 1e-12


def test_prepare_compiles_before_the_first_apply(engine, port):
    # kt_sv_prepare compiles a circuit's block kernels up front; an apply of the
    # same structure with other angles then runs them at once, and a plan
    # served from the plan cache takes the new angles
    old = {k: capi.tuning_get(k) for k in ("fused_jit", "jit_min_qubits", "jit_after")}
    try:
        capi.tuning_set("fused_jit", 2)
        capi.tuning_set("jit_min_qubits", 17)
        capi.tuning_set("jit_after", 0)
        n = 17
        gates, params = W.hea(n, 3, seed=61)
        sv = capi.Statevector(n)
        k0 = capi.jit_stats()["kernels"]
        sv.prepare(gates, params)
        s1 = capi.jit_stats()
        assert s1["kernels"] > k0
        for shift in (0.0, 0.41, -1.3):
            p = params + shift
            sv.set_basis(0)
            sv.apply(gates, p)
            assert np.abs(sv.download() - port.apply(n, basis(n), gates, p)).max() < 1e-12
        s2 = capi.jit_stats()
        assert s2["kernels"] == s1["kernels"] and s2["launches"] > s1["launches"]
        sv.close()
    finally:
        for k, v in old.items():
            capi.tuning_set(k, v)


def test_scaled_ops(jit, port):
    # jit_scale_ops: uncontrolled H / RY / RX run divided by their m00, the
    # block's product of those factors applied once (by another gate of the
    # block, or before the store); the same state as the unscaled kernels
    n = 18
    init = random_state(n, 71)
    g = W.random_layers(n, 4, seed=71, mixed=True)
    a = _apply(n, init, g)
    capi.tuning_set("jit_scale_ops", 0)
    b = _apply(n, init, g)
    capi.tuning_set("jit_scale_ops", 1)
    assert np.abs(a - b).max() < 1e-13
    assert np.abs(a - port.apply(n, init, g)).max() < 1e-12
    # only H, RY and CX: no gate of a block takes the factor, it has its own slot
    recs = []
    for layer in range(6):
        recs += [W.gate("H" if (q + layer) % 2 else "RY", q, angle=0.3 + q) for q in range(n)]
        recs += [W.gate("CX", q + 1, control=q) for q in range(layer % 2, n - 1, 2)]
    g2 = np.concatenate(recs)
    s0 = capi.jit_stats()
    got = _apply(n, init, g2)
    assert capi.jit_stats()["launches"] > s0["launches"]
    assert np.abs(got - port.apply(n, init, g2)).max() < 1e-12


def test_scaled_ops_out_of_range_fall_back(jit, port):
    # RY(pi) has m00 = cos(pi / 2) ~ 6e-17: twelve in one block take the
    # factor below 1e-150, so that apply runs on the precompiled kernels
    n = 16
    rng = np.random.default_rng(72)
    recs = [W.gate("RY", q % 6, angle=np.pi) for q in range(12)] + [W.gate("U", 2, u=W.haar_unitary2(rng))]
    g = np.concatenate(recs)
    init = random_state(n, 72)
    assert capi.plan_stats(n, g)["blocks"] == 1
    s0 = capi.jit_stats()
    got = _apply(n, init, g)
    assert capi.jit_stats()["launches"] == s0["launches"]
    assert np.abs(got - port.apply(n, init, g)).max() < 1e-12
    # the same structure with ordinary angles runs the compiled blocks
    g["angle"][:12] = rng.uniform(0.2, 2.0, 12)
    got = _apply(n, init, g)
    assert capi.jit_stats()["launches"] > s0["launches"]
    assert np.abs(got - port.apply(n, init, g)).max() < 1e-12


@pytest.mark.parametrize("knobs", [
    {"jit_tma": 1},
    {"jit_tma": 1, "jit_tma_stages": 2},
    {"jit_tma": 1, "jit_tma_stages": 4, "fused_tile_bits": 11},
    {"jit_tma": 1, "fused_reg_bits": 3},
    {"jit_tma": 1, "jit_tma_ctas": 2, "fused_tile_bits": 11, "fused_reg_bits": 3},
    {"jit_tma": 1, "jit_tma_ctas": 2, "fused_tile_bits": 11},
])
@pytest.mark.parametrize("n,layers,seed", [(13, 4, 81), (18, 4, 82), (22, 3, 83)])
def test_tma_blocks_match_oracle(jit, port, knobs, n, layers, seed):
    """TMA-pipelined compiled blocks (tiles moved by tensor copies into
    swizzled stage buffers, a producer warp, one tile group per CTA, one or
    two CTAs per SM): the oracle's amplitudes; from 13 qubits (two tiles) to 22 (every tile
    shape the planner makes, including tiles with more than four runs)."""
    old = {k: capi.tuning_get(k) for k in knobs}
    try:
        for k, v in knobs.items():
            capi.tuning_set(k, v)
        g = W.random_layers(n, layers, seed=seed, mixed=True)
        init = random_state(n, seed)
        s0 = capi.jit_stats()
        got = _apply(n, init, g)
        s1 = capi.jit_stats()
        assert not s1["failed"] and s1["launches"] > s0["launches"]
        assert np.abs(got - port.apply(n, init, g)).max() < 1e-12
        capi.tuning_set("jit_tma", 0)
        ref = _apply(n, init, g)
        assert np.abs(got - ref).max() < 1e-13
    finally:
        for k, v in old.items():
            capi.tuning_set(k, v)


def test_tma_blocks_at_26_qubits(jit):
    """The bench circuit family at 26 qubits (1 GiB): TMA blocks equal the
    classic compiled blocks."""
    n = 26
    g = W.random_layers(n, 4, seed=84, mixed=True)
    old = capi.tuning_get("jit_tma")
    try:
        capi.tuning_set("jit_tma", 1)
        a = _apply(n, basis(n), g)
        capi.tuning_set("jit_tma", 0)
        b = _apply(n, basis(n), g)
    finally:
        capi.tuning_set("jit_tma", old)
    assert np.abs(a - b).max() < 1e-13
