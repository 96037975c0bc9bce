"""Cubins from the on-disk cache (KT_JIT_CACHE_DIR) load and run: two fresh
processes prepare and apply the same 16-qubit circuit, and create and
evaluate the same 8-instance batch (13-14 qubits: compiled plan-structure
classes), with the cache on.  The first compiles with NVRTC and fills the
directory; the second runs NVRTC not once, takes every program from the
directory, launches the compiled blocks, and gives bit-identical amplitudes
(which match the oracle, 1e-12), energies and gradients."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import basis
from kettle_b200 import workloads as W

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

SCRIPT = """
import json, sys
import numpy as np
from kettle_b200 import capi
from kettle_b200 import workloads as W
n = 16
g = W.random_layers(n, 4, seed=11, mixed=True)
sv = capi.Statevector(n)
sv.prepare(g)
sv.apply(g)
np.save(sys.argv[1], sv.download())
circuits, params = W.hea_batch(8, seed=3, qubits=(13, 14), layers=(2, 3), n_strings=6)
items, gates, strings, coeffs, n_params = capi.batch_items(circuits)
b = capi.Batch(items, gates, strings, coeffs, n_params)
e, grad = b.evaluate(params)
classes = b.stats()["compiled_classes"]
b.close()
np.save(sys.argv[1] + ".batch.npy", np.concatenate([e, grad]))
print(json.dumps({**capi.jit_cache_stats(), "launches": capi.jit_stats()["launches"], "classes": classes}))
"""


def _run(cache, out):
    env = dict(os.environ, KT_JIT_CACHE_DIR=str(cache), PYTHONPATH=str(ROOT))
    r = subprocess.run([sys.executable, "-c", SCRIPT, str(out)], env=env, cwd=str(ROOT), capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_cached_cubins_run_in_a_new_process(engine, port, tmp_path):
    cache = tmp_path / "cubins"
    cache.mkdir()
    first = _run(cache, tmp_path / "a.npy")
    assert first["nvrtc_compiles"] >= 2 and first["disk_hits"] == 0 and first["launches"] > 0
    assert first["classes"] >= 1
    assert any(p.suffix == ".cubin" for p in cache.iterdir())
    second = _run(cache, tmp_path / "b.npy")
    assert second["nvrtc_compiles"] == 0 and second["disk_hits"] == first["nvrtc_compiles"]
    assert second["launches"] > 0
    a, b = np.load(tmp_path / "a.npy"), np.load(tmp_path / "b.npy")
    assert np.array_equal(a, b)
    assert np.array_equal(np.load(tmp_path / "a.npy.batch.npy"), np.load(tmp_path / "b.npy.batch.npy"))
    n = 16
    want = port.apply(n, basis(n), W.random_layers(n, 4, seed=11, mixed=True))
    assert np.abs(b - want).max() < 1e-12
