"""The C-ABI library loads and exports every symbol include/kettle_b200.h
declares; host-only helpers work without a GPU; device calls on a machine
without a GPU fail with a status and a message instead of crashing."""
import re

import numpy as np
import pytest

from conftest import ROOT
from kettle_b200 import capi


def _declared():
    text = (ROOT / "include" / "kettle_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kt_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    declared = _declared()
    assert len(declared) >= 38
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert sorted(capi.exported_symbols()) == _declared()


def test_record_layouts():
    assert capi.GATE_DTYPE.itemsize == 88
    assert capi.PAULI_DTYPE.itemsize == 24
    assert capi.GATE_DTYPE.fields["angle"][1] == 16
    assert capi.GATE_DTYPE.fields["u"][1] == 24


def test_version_and_error_strings():
    assert capi.lib().kt_version() >= 100
    # a bad argument is rejected on the host, before any device work
    with pytest.raises(capi.KettleError) as e:
        capi.pairs_single(3, 5)
    assert "target" in str(e.value)


def test_no_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(capi.KettleError) as e:
        capi.Statevector(4)
    assert e.value.code in (-2, -3)


def test_canonicals_helper_is_host_only():
    v = capi.canonicals_mt19937(5489, 10)
    assert np.all((v >= 0) & (v < 1))


def test_batch_rejects_bad_items_on_the_host():
    from kettle_b200 import workloads as W
    g, p = W.hea(4, 1, seed=0)
    s, c = W.random_paulis(4, 3, seed=0)
    items, gates, strings, coeffs, n_params = capi.batch_items([(4, g, p.size, s, c)])
    bad = items.copy()
    bad["n_params"] = p.size + 1          # parameter range past the end of params
    with pytest.raises(capi.KettleError) as e:
        capi.Batch(bad, gates, strings, coeffs, n_params)
    assert e.value.code == -1 and "out of range" in str(e.value)
    wide = strings.copy()
    wide["z"][0] = 1 << 6                  # a Pauli string on a qubit the item does not have
    with pytest.raises(capi.KettleError) as e:
        capi.Batch(items, gates, wide, coeffs, n_params)
    assert "outside its qubits" in str(e.value)
    slot = gates.copy()
    slot["param"][0] = 99                  # a gate bound to a slot the item does not have
    with pytest.raises(capi.KettleError) as e:
        capi.Batch(items, slot, strings, coeffs, n_params)
    assert "parameter slot 99" in str(e.value)
    meas = np.concatenate([gates, W.gate("M", 0)])
    items2, _, _, _, _ = capi.batch_items([(4, meas, p.size, s, c)])
    with pytest.raises(capi.KettleError) as e:
        capi.Batch(items2, meas, strings, coeffs, n_params)
    assert "M gates" in str(e.value)


def test_run_time_block_kernels_compile_on_the_host():
    # the generated straight-line block kernels compile for sm_100a with NVRTC
    # (no GPU needed: compile only, nothing is loaded)
    from kettle_b200 import workloads as W
    g = W.random_layers(14, 3, seed=1, mixed=True)
    assert capi.jit_compile_only(14, g) >= 1
    gates, params = W.hea(13, 2, seed=2)
    assert capi.jit_compile_only(13, gates, params) >= 1
    assert capi.jit_compile_only(15, W.random_layers(15, 2, seed=3, mixed=True),
                                 dtype=capi.KT_C64) >= 1


@pytest.mark.parametrize("knobs", [
    {"jit_async_load": 1}, {"fused_reg_bits": 3}, {"jit_fence": 2, "jit_merge_diag": 0},
    {"jit_skip_io": 0, "jit_prefetch": 0, "fused_tile_bits": 11}, {"jit_scale_ops": 0}, {"jit_remat": 0},
])
def test_generated_kernel_variants_compile_on_the_host(knobs):
    from kettle_b200 import workloads as W
    old = {k: capi.tuning_get(k) for k in knobs}
    try:
        for k, v in knobs.items():
            capi.tuning_set(k, v)
        g = W.random_layers(14, 2, seed=5, mixed=True)
        assert capi.jit_compile_only(14, g) >= 1
        assert capi.jit_compile_only(15, g, dtype=capi.KT_C64) >= 1
    finally:
        for k, v in old.items():
            capi.tuning_set(k, v)


def test_scaled_block_without_a_sink_compiles_on_the_host():
    # a block of only H, RY and CX has scaled gates and no unscaled gate to
    # take their factor: the generated kernel applies it before the store
    from kettle_b200 import workloads as W
    n = 14
    recs = []
    for layer in range(3):
        recs += [W.gate("H" if (q + layer) % 2 else "RY", q, angle=0.4 + q) for q in range(n)]
        recs += [W.gate("CX", q + 1, control=q) for q in range(layer % 2, n - 1, 2)]
    assert capi.jit_compile_only(n, np.concatenate(recs)) >= 1


def test_jit_dump_writes_source_and_register_summary(tmp_path, monkeypatch):
    # KT_JIT_DUMP_DIR (inspection): each generated program's source and
    # ptxas's register / spill summary of its kernels
    from kettle_b200 import workloads as W
    monkeypatch.setenv("KT_JIT_DUMP_DIR", str(tmp_path))
    assert capi.jit_compile_only(14, W.random_layers(14, 2, seed=9, mixed=True)) >= 1
    src = (tmp_path / "kt_jit_0.cu").read_text()
    log = (tmp_path / "kt_jit_0.log").read_text()
    assert "__global__" in src
    assert re.search(r"Used \d+ registers", log) and "spill" in log


def test_every_documented_knob_is_known_with_its_documented_default():
    # the knob list in include/kettle_b200.h against the library, in a fresh
    # process (no KT_TUNING): every name is accepted, and where the comment
    # states a default "(v)" after the range, kt_tuning_get returns it
    import subprocess
    import sys
    head = (ROOT / "include" / "kettle_b200.h").read_text()
    block = head[head.index("Launch-shape knobs of the engine"):head.index("Unknown names return")]
    rows = re.findall(r"^ \*   ([a-z_0-9]+) +(\d+(?:\.\.[0-9e]+| or \d+|, \d+, \d+)?) +(?:\((\d+)\))?", block, re.M)
    assert len(rows) >= 20 and all(r[2] for r in rows)
    names = [r[0] for r in rows]
    code = ("import json, sys\nsys.path.insert(0, %r)\nfrom kettle_b200 import capi\n"
            "print(json.dumps({n: capi.tuning_get(n) for n in %r}))" % (str(ROOT), names))
    env = {k: v for k, v in __import__("os").environ.items() if k != "KT_TUNING"}
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, check=True)
    got = __import__("json").loads(out.stdout.strip().splitlines()[-1])
    for name, _, default in rows:
        if default:
            assert got[name] == int(default), (name, got[name], default)


def test_adjoint_blocks_compile_on_the_host():
    # adjoint_jit = 1: kt_jit_compile_only compiles the fused adjoint blocks of
    # the circuit's backward sweep (complex128 and complex64)
    from kettle_b200 import workloads as W
    old = capi.tuning_get("adjoint_jit")
    try:
        capi.tuning_set("adjoint_jit", 1)
        g, p = W.hea(14, 3, seed=3)
        mixed = W.random_layers(13, 2, seed=4, mixed=True)
        mixed["param"][::3] = np.arange(mixed[::3].size)
        mp = np.linspace(0.1, 2.0, mixed[::3].size)
        assert capi.jit_compile_only(14, g, p) >= 1
        assert capi.jit_compile_only(13, mixed, mp) >= 1
        assert capi.jit_compile_only(13, mixed, mp, dtype=capi.KT_C64) >= 1
    finally:
        capi.tuning_set("adjoint_jit", old)
